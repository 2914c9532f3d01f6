"""Autotuner for the direct J/K plan: per angular-momentum class, the
primitive-quartet chunk of a work item (2 .. 128), and the number of
streams the class launches share.

    python -m pyquante_b200.autotune [--mode fp64|mixed] [--out PATH]   # (H2O)8 / 6-31G** on cuda:0

The objective is the whole Fock-build time (CUDA events, median of 5,
after an L2 flush): the class kernels run concurrently on several streams,
so per-class latency is the wrong target.  A global chunk sweep is followed
by per-class coordinate descent (heaviest classes first) and a stream-count
sweep.
Results are stored as JSON (``tuned.json`` next to this file) and applied
by ``BasisEngine`` when present.
"""
import ctypes
import json
import os

import numpy as np

TUNED = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned.json")
CHUNKS = (2, 4, 8, 16, 32, 64, 128)


def load():
    if os.path.exists(TUNED):
        with open(TUNED) as f:
            return json.load(f)
    return None


def apply(eng, tuned=None):
    """Set the tuned knobs on a BasisEngine's context (before its plan)."""
    from . import _lib
    tuned = tuned if tuned is not None else load()
    if not tuned:
        return False
    for qc, ch in enumerate(tuned.get("chunk", [])):
        eng.ctx.check(eng.ctx.lib.pqb_set_param(eng.ctx.h, _lib.PQB_PARAM_CHUNK, qc, int(ch)))
    if "streams" in tuned:
        eng.ctx.check(eng.ctx.lib.pqb_set_param(eng.ctx.h, _lib.PQB_PARAM_STREAMS, 0, int(tuned["streams"])))
    if "order" in tuned:
        eng.ctx.check(eng.ctx.lib.pqb_set_param(eng.ctx.h, _lib.PQB_PARAM_ORDER, 0, int(tuned["order"])))
    return True


def _build_ms(eng, D, J, K, mode, schwarz, fp32_threshold, flush, reps=5):
    import torch
    ts = []
    for _ in range(reps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        eng.jk(D, mode, schwarz, fp32_threshold, J=J, K=K)
        e1.record()
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    return float(np.median(ts))


def tune(eng, D, mode="mixed", schwarz=1e-12, fp32_threshold=1e-5, verbose=True):
    """Coordinate descent on the whole Fock-build time (the class kernels run
    concurrently, so a class's own latency is the wrong objective)."""
    import torch
    from . import _lib
    J = torch.zeros_like(D)
    K = torch.zeros_like(D)
    flush = torch.empty(64 << 20, dtype=torch.float32, device=D.device)
    lib, h = eng.ctx.lib, eng.ctx.h

    order = 1

    def evaluate(chunk, streams):
        for qc, ch in enumerate(chunk):
            eng.ctx.check(lib.pqb_set_param(h, _lib.PQB_PARAM_CHUNK, qc, int(ch)))
        eng.ctx.check(lib.pqb_set_param(h, _lib.PQB_PARAM_STREAMS, 0, int(streams)))
        eng.ctx.check(lib.pqb_set_param(h, _lib.PQB_PARAM_ORDER, 0, int(order)))
        eng._plan_key = None
        eng.plan(schwarz, fp32_threshold)
        return _build_ms(eng, D, J, K, mode, schwarz, fp32_threshold, flush)

    streams = 8
    best_t, best_ch = None, None
    for ch in CHUNKS:                                   # one chunk for every class
        t = evaluate([ch] * 21, streams)
        if verbose:
            print("chunk %3d everywhere: %.4f ms" % (ch, t))
        if best_t is None or t < best_t:
            best_t, best_ch = t, ch
    chunk = [best_ch] * 21
    qa = (ctypes.c_int64 * 42)()
    pa = (ctypes.c_int64 * 42)()
    eng.ctx.check(lib.pqb_plan_stats(h, qa, pa))
    cost = np.array(pa[:]).reshape(2, 21).sum(axis=0)
    for qc in np.argsort(-cost):                        # per class, heaviest first
        if cost[qc] == 0:
            continue
        for ch in CHUNKS:
            if ch == chunk[qc]:
                continue
            trial = list(chunk)
            trial[qc] = ch
            t = evaluate(trial, streams)
            if t < 0.99 * best_t:
                best_t, chunk = t, trial
    for ns in (2, 4, 8, 12, 16):
        t = evaluate(chunk, ns)
        if t < 0.99 * best_t or (ns == streams and t < best_t):
            best_t, streams = t, ns
    times = {}
    for od in (0, 1):
        order = od
        times[od] = evaluate(chunk, streams)
        if verbose:
            print("order %d: %.4f ms" % (od, times[od]))
    order = min(times, key=times.get)
    best_t = min(best_t, times[order])
    evaluate(chunk, streams)
    result = {"chunk": [int(c) for c in chunk], "streams": int(streams), "order": int(order), "build_ms": best_t,
              "mode": mode,
              "workload": "(H2O)8 6-31G** seed 0"}
    if verbose:
        print(json.dumps(result))
    return result


def main():
    import argparse

    import torch
    from . import Ints, geometries
    from .Basis.basis import BasisSet
    from .LA2 import geigh, mkdens
    from .engine import BasisEngine
    mol = geometries.water_cluster(8, seed=0)
    bs = BasisSet(mol, "6-31g**")
    eng = BasisEngine(bs.bfs)
    eng.plan()
    S, h = Ints.get1ints(bs, mol)
    _, C = geigh(torch.as_tensor(h, device="cuda"), torch.as_tensor(S, device="cuda"))
    D = mkdens(C, 0, mol.get_nel() // 2).contiguous()
    ap = argparse.ArgumentParser()
    ap.add_argument("--mode", default="fp64", choices=["fp64", "mixed"], help="build to tune (default: FP64)")
    ap.add_argument("--out", default=TUNED, help="where to write the result (default: tuned.json here)")
    a = ap.parse_args()
    res = tune(eng, D, mode=a.mode)
    with open(a.out, "w") as f:
        json.dump(res, f, indent=1)
    print("wrote", a.out)


if __name__ == "__main__":
    main()
