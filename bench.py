"""Benchmark: integral-direct 2J-K Fock build on (H2O)8 / 6-31G** (N = 200).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl pqb|reference]
                    [--no-cpu-baseline] [--workload h2o8|stored|c16h34|h2o4-grad|batch|mp2|dft]

One step = one full FP64 2J-K Fock build G(D) = 2J(D) - K(D) for a fixed SCF
density D of the seeded (H2O)8 cluster (Schwarz 1e-12).  value = nominal
unique quartets Q = P(P+1)/2 (P = N(N+1)/2, 202,015,050) per second of Fock
build, the count the reference's get2ints evaluates (PyQuante/Ints.py:146-167);
the line also gives the quartets computed after Schwarz screening per second.
The mixed FP32/FP64 build (quartets with Q_ab Q_cd < 1e-5 in FP32) is timed
beside it, with its SCF energy error against the FP64 path.  Under torchrun
the quartet lists are sharded over ranks and J/K summed with one NCCL
all-reduce per build (strong scaling).

The reference arm (--impl reference) times the reference's own C Rys engine
(oracle/_ref, compiled from the reference's Src/lib/utils/crys.c) over a
bounded sample of the same quartets on all host cores and on one, plus full
get2ints + get2JmK steps of small molecules.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "(H2O)8 cluster, 6-31G** cartesian, N=200, seed 0, 9 A cube"
SCHWARZ = 1e-12
FP32_THRESH = 1e-5
L2_FLUSH_BYTES = 256 << 20
# DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum) of one stored-integral J/K
# launch on this workload, and summed over the 21 class launches of one FP64 direct build
STORED_TRAFFIC_BYTES = 1620658000 + 5230080
DIRECT_TRAFFIC_BYTES = 34722560 + 0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="pqb", choices=["pqb", "reference"])
    p.add_argument("--precision", default="fp64", choices=["mixed", "fp64"],
                   help="precision of the --profile-builds builds")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-graph", action="store_true", help="launch the timed builds eagerly instead of replaying "
                                                             "a captured CUDA graph")
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--soak", type=int, default=3000, help="untimed builds run under the clock sampler before the "
                                                           "timed ones")
    p.add_argument("--workload", default="h2o8", choices=["h2o8", "stored", "c16h34", "h2o4-grad", "batch", "mp2", "dft"],
                   help="h2o8: the headline Fock build; the others are the secondary workloads "
                        "(C16H34 threshold sweep, (H2O)4 gradient, batched SCF)")
    p.add_argument("--batch-count", type=int, default=512)
    p.add_argument("--single-sample", type=int, default=64)
    p.add_argument("--profile-builds", type=int, default=0,
                   help="run this many untimed Fock builds after setup and exit (for ncu captures)")
    return p.parse_args()


def molecule():
    from pyquante_b200 import geometries
    return geometries.water_cluster(8, seed=0)


def nominal_quartets(n):
    P = n * (n + 1) // 2
    return P * (P + 1) // 2


# ------------------------------------------------------------ CPU reference --
def _oracle_table(bs):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyq_oracle as O
    if bs is None:
        return O, None
    return O, O.Table([O.BF(bf.origin, bf.powers, list(zip(bf.pexps, bf.pcoefs))) for bf in bs.bfs])


def reference_rate(bs, seconds, seed=0, nproc=None):
    """Quartets/s of the reference's compiled Rys engine (ref_fock, forked
    workers over bra rows) on a bounded random sample of bra rows."""
    O, tab = _oracle_table(bs)
    exe = os.path.join(ROOT, "oracle", "_ref", "ref_fock")
    if not os.path.exists(exe):
        raise RuntimeError("oracle/_ref/ref_fock not built (make -C oracle ref)")
    nproc = nproc or os.cpu_count() or 1
    n = tab.nbf
    P = n * (n + 1) // 2
    rng = np.random.default_rng(seed)
    with tempfile.TemporaryDirectory() as td:
        bpath = os.path.join(td, "basis.bin")
        tab.write(bpath)

        def run(nrows):
            rows = np.sort(rng.choice(P, size=nrows, replace=False)).astype(np.int64)
            rpath = os.path.join(td, "rows.bin")
            rows.tofile(rpath)
            out = subprocess.run([exe, bpath, rpath, str(nproc)], capture_output=True, text=True, check=True)
            return json.loads(out.stdout)

        probe = run(max(nproc, 4))
        rate = probe["quartets"] / max(probe["seconds"], 1e-6)
        avg_row = nominal_quartets(n) / P
        nrows = int(min(P, max(nproc, rate * seconds / avg_row)))
        r = run(nrows)
    return dict(value=r["quartets"] / r["seconds"], quartets=r["quartets"], seconds=r["seconds"], rows=nrows,
                cores=nproc)


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def reference_full_steps(nproc):
    """Full reference steps, timed: Ints.get2ints (every unique quartet) and
    one get2JmK on the packed array, through the reference's compiled crys
    (ref_fock.c), for water / STO-3G (406 quartets) and water clusters of
    two and three molecules in 6-31G** (N = 50, 75)."""
    O, _ = _oracle_table(None)
    from pyquante_b200 import geometries
    from pyquante_b200.Basis.p631ss import basis_data as P631SS
    from pyquante_b200.Basis.sto3g import basis_data as STO3G
    lib = O.ref_lib("fock")
    out = []
    for name, mol, basis in (("water / STO-3G", geometries.water(), STO3G),
                             ("(H2O)2 / 6-31G**", geometries.water_cluster(2, seed=4), P631SS),
                             ("(H2O)3 / 6-31G**", geometries.water_cluster(3, seed=2), P631SS)):
        bfs = O.build_basis([(at.atno, tuple(at.r)) for at in mol.atoms], basis)
        t = O.Table(bfs)
        nq = O.nquartets(t.nbf)
        ints = np.zeros(nq)
        rng = np.random.default_rng(0)
        C = rng.standard_normal((t.nbf, max(1, t.nbf // 5)))
        D = np.ascontiguousarray(C @ C.T)
        G = np.zeros_like(D)
        t0 = time.perf_counter()
        rc = lib.ref_get2ints(*t.args(), ints.ctypes.data_as(O._dp), nproc)
        t1 = time.perf_counter()
        lib.ref_get2JmK(t.nbf, ints.ctypes.data_as(O._dp), D.ctypes.data_as(O._dp), G.ctypes.data_as(O._dp))
        t2 = time.perf_counter()
        if rc != 0:
            raise RuntimeError("ref_get2ints failed (%d)" % rc)
        out.append({"molecule": name, "nbf": t.nbf, "quartets": nq, "get2ints_s": t1 - t0, "get2JmK_s": t2 - t1,
                    "step_s": t2 - t0, "quartets_per_s": nq / (t1 - t0), "processes": nproc})
    return out


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from pyquante_b200.Basis.basis import BasisSet
    bs = BasisSet(molecule(), "6-31g**")
    cores = os.cpu_count() or 1
    per_step = max(2.0, min(20.0, 120.0 / max(a.steps + a.warmup, 1)))
    for i in range(a.warmup):
        reference_rate(bs, per_step / 2, seed=100 + i, nproc=cores)
    secs, counts = [], []
    for i in range(a.steps):
        r = reference_rate(bs, per_step, seed=i, nproc=cores)
        secs.append(r["seconds"])
        counts.append(r["quartets"])
    value = sum(counts) / sum(secs)
    one = reference_rate(bs, min(per_step, 10.0), seed=1000, nproc=1)
    full = reference_full_steps(cores)
    Q = nominal_quartets(len(bs))
    line = {
        "impl": "reference", "metric": "ERI quartets/s (2J-K Fock build, FP64; nominal unique (ij|kl))",
        "value": value, "unit": "quartets/s", "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1e3 * sum(secs) / len(secs), "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "precision": "fp64", "nominal_quartets": Q,
                   "step": "one bounded sample of the workload: random bra rows of Ints.get2ints, every kl >= ij "
                           "per row, ~%.0f s on all host cores (ms_per_step is that sample's time)" % per_step},
        "full_build_s_extrapolated": Q / value, "extrapolated": True,
        "extrapolation_note": "the reference computes every unique quartet unscreened; a full c1 build at the "
                              "sampled rate would take full_build_s_extrapolated seconds",
        "one_process": {"value": one["value"], "unit": "quartets/s", "quartets": one["quartets"],
                        "seconds": one["seconds"]},
        "full_steps": full,
        "cpu_model": _cpu_model(),
        "cpu_baseline": {"value": value, "unit": "quartets/s", "cores": cores, "kind": "reference",
                         "sample": "%d quartets over %d steps" % (sum(counts), a.steps)},
        "e2e": {"value": value, "unit": "quartets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ------------------------------------------------------------------- clocks --
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._th = None

    def __enter__(self):
        def loop():
            while not self._stop.is_set():
                try:
                    out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                         timeout=5).stdout.strip()
                    if out:
                        self.rows.append([c.strip() for c in out.split(",")])
                except Exception:
                    pass
                self._stop.wait(0.2)
        self._th = threading.Thread(target=loop, daemon=True)
        self._th.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._th.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# --------------------------------------------------------------- GPU arm --
# --------------------------------------------------- secondary workloads --
def measured_hbm_gbs():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (measured)"
    except Exception:
        return 6650.0, "fallback 6.65 TB/s"


def run_stored(a):
    """Stored-integral 2J-K (PyQuante/Ints.py:225-238) on (H2O)8 / 6-31G**:
    the packed array (Q doubles, 1.6 GB) is built once, then each step is
    one pqb_jk_packed over it.  Algorithmic bytes per build: 8 Q + 3 * 8 N^2
    (D in, J and K out).  The packed array is 13x the L2, so no flush."""
    import torch

    from pyquante_b200 import Ints
    from pyquante_b200.Basis.basis import BasisSet
    from pyquante_b200.engine import BasisEngine, jk_packed
    mol = molecule()
    bs = BasisSet(mol, "6-31g**")
    n = len(bs)
    eng = BasisEngine(bs.bfs)
    ints = eng.eri_packed()
    # a dense symmetric density of the cluster's rank (seeded), so every
    # J/K contribution is nonzero and takes its atomics
    nocc = mol.get_nel() // 2
    C = np.linalg.qr(np.random.default_rng(0).standard_normal((n, nocc)))[0]
    D = torch.as_tensor(C @ C.T, device="cuda")
    for _ in range(a.warmup):
        jk_packed(ints, D, eng.ctx)
    torch.cuda.synchronize()
    ts = []
    for _ in range(a.steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        jk_packed(ints, D, eng.ctx)
        e1.record()
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    ms = float(np.mean(ts))
    Q = ints.numel()
    nbytes = 8 * Q + 3 * 8 * n * n
    peak, src = measured_hbm_gbs()
    gbs = nbytes / (ms * 1e-3) / 1e9
    print(json.dumps({"metric": "stored-integral 2J-K build (get2JmK on packed Ints)", "value": Q / (ms * 1e-3),
                      "unit": "integrals/s", "ms_per_step": ms, "steps": a.steps, "warmup": a.warmup,
                      "data": "synthetic", "dtype": "f64",
                      "config": {"workload": WORKLOAD, "packed_integrals": Q, "bytes_per_build": nbytes,
                                 "l2": "packed array 1.6 GB > L2, no flush"},
                      "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s",
                                   "frac": gbs / peak, "traffic": STORED_TRAFFIC_BYTES, "peak_source": src,
                                   "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch",
                                   "kernel": "jk_packed_reg_kernel<7>"}}))

def run_c16h34(a):
    """C16H34 / 6-31G* (N = 308): FP64 vs mixed Fock build and SCF energy for
    FP32 thresholds 1e-7 .. 1e-4 (Schwarz 1e-12)."""
    import torch

    from pyquante_b200 import geometries
    from pyquante_b200.Basis.basis import BasisSet
    from pyquante_b200.engine import BasisEngine
    from pyquante_b200.hartree_fock import rhf
    mol = geometries.alkane(16)
    bs = BasisSet(mol, "6-31g*")
    n = len(bs)
    out = {"workload": "all-trans C16H34, 6-31G* cartesian, N=%d" % n, "nominal_quartets": nominal_quartets(n)}
    e64, _, orbs = rhf(mol, bfs=bs, direct=True, precision="fp64", ConvCriteria=1e-9, MaxIter=60, DoAveraging=True)
    out["energy_fp64"] = e64
    eng = bs._pqb_engine
    # the builds are timed on the converged FP64 density
    Cocc = torch.as_tensor(np.asarray(orbs.cpu() if hasattr(orbs, "cpu") else orbs)[:, :mol.get_nel() // 2],
                           dtype=torch.float64, device="cuda")
    D = (Cocc @ Cocc.T).contiguous()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def time_build(mode, thr):
        for _ in range(a.warmup):
            eng.jk(D, mode, SCHWARZ, thr)
        ts = []
        for _ in range(a.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            eng.jk(D, mode, SCHWARZ, thr)
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return float(np.median(ts))

    out["fp64_ms_per_build"] = time_build("fp64", 1e-5)
    sweep = []
    for thr in (1e-7, 1e-6, 1e-5, 1e-4):
        em, _, _ = rhf(mol, bfs=bs, direct=True, precision="mixed", fp32_threshold=thr, ConvCriteria=1e-9,
                       MaxIter=60, DoAveraging=True)
        ms = time_build("mixed", thr)
        c = eng.plan_counts
        sweep.append({"fp32_threshold": thr, "energy": em, "abs_dE": abs(em - e64), "ms_per_build": ms,
                      "speedup_vs_fp64": out["fp64_ms_per_build"] / ms, "kept_fp64": c["fp64"], "kept_fp32": c["fp32"]})
    out["sweep"] = sweep
    print(json.dumps({"metric": "C16H34 mixed-precision threshold sweep", "unit": "ms/Fock build, Eh",
                      "config": out, "data": "synthetic"}))


def run_h2o4_grad(a):
    """(H2O)4 / 6-31G* perturbed +-0.05 bohr (seed 7): analytic gradient,
    FP64 and mixed, against central finite differences (step 1e-4 bohr)."""
    from pyquante_b200 import geometries
    from pyquante_b200.Molecule import Molecule
    from pyquante_b200.force import rhf_with_gradient
    from pyquante_b200.hartree_fock import rhf
    mol = geometries.perturbed(geometries.water_cluster(4, seed=0), 0.05, seed=7)
    opts = dict(ConvCriteria=1e-11, MaxIter=200, DoAveraging=True)
    res = {}
    for prec in ("fp64", "mixed"):
        rhf_with_gradient(mol, "6-31g*", precision=prec, **opts)          # warm-up
        t0 = time.perf_counter()
        e, g, _, _ = rhf_with_gradient(mol, "6-31g*", precision=prec, **opts)
        res[prec] = (e, g, time.perf_counter() - t0)
    h = 1e-4
    fd = np.zeros_like(res["fp64"][1])
    atoms = [(at.atno, tuple(at.r)) for at in mol.atoms]
    for i in range(len(atoms)):
        for x in range(3):
            vals = []
            for d in (h, -h):
                r = list(atoms[i][1])
                r[x] += d
                at2 = list(atoms)
                at2[i] = (atoms[i][0], tuple(r))
                vals.append(rhf(Molecule("m", at2, units="bohr"), basis_data="6-31g*", **opts)[0])
            fd[i, x] = (vals[0] - vals[1]) / (2 * h)
    print(json.dumps({"metric": "(H2O)4 RHF gradient error vs central differences", "unit": "Eh/bohr",
                      "data": "synthetic",
                      "config": {"workload": "(H2O)4 6-31G*, N=76, +-0.05 bohr perturbation seed 7",
                                 "fp64_max_err": float(np.abs(res["fp64"][1] - fd).max()),
                                 "mixed_max_err": float(np.abs(res["mixed"][1] - fd).max()),
                                 "mixed_vs_fp64_energy": abs(res["mixed"][0] - res["fp64"][0]),
                                 "fp64_scf_plus_gradient_s": res["fp64"][2],
                                 "mixed_scf_plus_gradient_s": res["mixed"][2]}}))


def run_batch(a):
    """512 water clusters, k ~ U{1..12}, basis 50/50 STO-3G / 6-31G*: one
    batched mixed-precision SCF (DIIS, conv 1e-8 plus a commutator test,
    densities by batched purification, each iteration one CUDA graph
    replay) vs a loop of single solves over a random sample."""
    from pyquante_b200 import geometries
    from pyquante_b200.batch import batched_rhf
    from pyquante_b200.hartree_fock import rhf
    systems = geometries.cluster_batch(a.batch_count, seed=0)
    batched_rhf(systems[:8], precision="mixed", conv=1e-8)          # warm-up (compile, allocator)
    res = batched_rhf(systems, precision="mixed", conv=1e-8, maxiter=80, graph=True)
    rng = np.random.default_rng(1)
    pick = rng.choice(len(systems), size=min(a.single_sample, len(systems)), replace=False)
    single = []
    for i in pick:
        mol, basis = systems[i]
        t0 = time.perf_counter()
        rhf(mol, basis_data=basis, direct=True, precision="mixed", ConvCriteria=1e-8, MaxIter=80, DoAveraging=True)
        dt = time.perf_counter() - t0
        # the energy to compare, from a single solve converged far below the
        # batch's criterion (rhf takes the energy from the DIIS-extrapolated
        # Fock matrix, as the reference does, which is not variational)
        e, _, _ = rhf(mol, basis_data=basis, direct=True, precision="mixed", ConvCriteria=1e-11, MaxIter=200,
                      DoAveraging=True)
        single.append((dt, abs(e - res["energies"][i])))
    st = np.array([s[0] for s in single])
    print(json.dumps({
        "metric": "batched RHF molecules/s", "value": len(systems) / res["scf_seconds"], "unit": "molecules/s",
        "data": "synthetic",
        "config": {"workload": "%d water clusters, k~U{1..12}, 50/50 STO-3G/6-31G*, seed 0" % len(systems),
                   "nbf_min_max": [int(res["nbf"].min()), int(res["nbf"].max())],
                   "converged": int(res["converged"].sum()), "iterations_max": int(res["iterations"].max()),
                   "scf_seconds": res["scf_seconds"], "setup_seconds": res["total_seconds"] - res["scf_seconds"],
                   "per_molecule_scf_s_p50": float(np.percentile(res["scf_times"], 50)),
                   "per_molecule_scf_s_p99": float(np.percentile(res["scf_times"], 99)),
                   "cuda_graph": res["graph"], "whole_iteration_graph": res["whole_iteration_graph"],
                   "incremental_fock_builds": res["incremental"],
                   "plan": res["plan"],
                   "single_solve_loop": {"sample": len(pick), "molecules_per_s": len(pick) / st.sum(),
                                         "p50_s": float(np.percentile(st, 50)), "p99_s": float(np.percentile(st, 99)),
                                         "max_abs_dE_vs_batched": float(max(s[1] for s in single))}}}))


def _timed(fn, steps, stream, flush):
    """Mean CUDA-event time (ms) of fn() on `stream`, L2 flushed before each."""
    import torch
    tot = 0.0
    for _ in range(steps):
        flush.zero_()          # L2 flush between timed builds, outside the timed window
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        tot += e0.elapsed_time(e1)
    return tot / steps


def _scf(mol, bs, precision, solver="eigh"):
    """RHF to 1e-10 Eh (DIIS) on the integral-direct path; returns the energy,
    the number of Fock builds and the wall time.  solver 'eigh': the
    reference's loop with the host eigensolver; 'purify': the loop on the
    GPU, densities by canonical purification, one eigensolve at the end."""
    from pyquante_b200 import Ints
    from pyquante_b200.hartree_fock import rhf

    class Counting(Ints.DirectInts):
        builds = 0

        def jk(self, D):
            Counting.builds += 1
            return super().jk(D)

    from pyquante_b200.Ints import _engine_for, get1ints
    eng = _engine_for(bs)
    S, h = get1ints(bs, mol)
    ints = Counting(eng, precision, SCHWARZ, FP32_THRESH)
    kw = dict(bfs=bs, integrals=(S, h, ints), ConvCriteria=1e-10, MaxIter=80, DoAveraging=True, solver=solver)
    rhf(mol, **kw)   # warm-up
    Counting.builds = 0
    t0 = time.perf_counter()
    e, _, _ = rhf(mol, **kw)
    if solver == "purify":
        import torch
        torch.cuda.synchronize()
    return e, Counting.builds, time.perf_counter() - t0


def run_mp2(a):
    """MP2 on (H2O)8 / 6-31G** (N = 200, 40 occupied orbitals): the AO -> MO
    transformation of the packed integrals (PyQuante/MP.py:20-97) timed on
    the device after the RHF, FP64 throughout."""
    import torch

    from pyquante_b200 import MP, Ints
    from pyquante_b200.Basis.basis import BasisSet
    from pyquante_b200.hartree_fock import rhf
    mol = molecule()
    bs = BasisSet(mol, "6-31g**")
    n = len(bs)
    nocc = mol.get_nel() // 2
    S, h, ints = Ints.getints(bs, mol)
    e, orbe, orbs = rhf(mol, bfs=bs, integrals=(S, h, ints), ConvCriteria=1e-10, MaxIter=80, DoAveraging=True)
    for _ in range(max(a.warmup, 1)):
        emp2 = MP.MP2(ints, orbs, orbe, nocc, n - nocc)
    torch.cuda.synchronize()
    ts = []
    for _ in range(a.steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        emp2 = MP.MP2(ints, orbs, orbe, nocc, n - nocc)
        e1.record()
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    ms = float(np.median(ts))
    nv = n - nocc
    P = n * (n + 1) // 2
    # GEMM flops of the two half-transformations (FMA = 2)
    fl = 2.0 * P * (n * n * nv + n * nocc * nv) + 2.0 * nocc * nv * (n * n * nocc + n * nocc * nv)
    print(json.dumps({"metric": "MP2 energy (AO->MO transform of packed Ints + pair energies)",
                      "value": ms, "unit": "ms", "higher_is_better": False, "steps": a.steps, "data": "synthetic",
                      "dtype": "f64",
                      "config": {"workload": WORKLOAD, "nocc": nocc, "nvirt": nv, "e_rhf": e, "e_mp2": emp2,
                                 "gemm_flops": fl, "gemm_tflops": fl / (ms * 1e-3) / 1e12,
                                 "path": "pqb_mo_unpack_rows/pairs + cuBLAS DGEMM (torch.matmul) + pqb_mp2_pairs"}}))


def run_dft(a):
    """SVWN DFT on (H2O)8 / 6-31G** (N = 200) with the reference's default
    grid (24 atoms x 32 x 194 points): one Coulomb-only direct build and one
    exchange-correlation build (density on the grid, functional, Fxc) timed
    on the device, and the whole SCF."""
    import torch

    from pyquante_b200 import Ints
    from pyquante_b200.Basis.basis import BasisSet
    from pyquante_b200.dft import dft, getXC
    from pyquante_b200.MolecularGrid import MolecularGrid
    mol = molecule()
    bs = BasisSet(mol, "6-31g**")
    t0 = time.perf_counter()
    e, orbe, orbs = dft(mol, bfs=bs, direct=True, ConvCriteria=1e-8, MaxIter=60)
    scf_s = time.perf_counter() - t0
    nocc = mol.get_nel() // 2
    C = torch.as_tensor(orbs, device="cuda")
    D = (C[:, :nocc] @ C[:, :nocc].T).contiguous()
    gr = MolecularGrid(mol)
    gr.set_bf_amps(bs.bfs)
    direct = Ints.get2ints(bs, direct=True)

    def xc():
        gr.setdens(D)
        return getXC(gr, mol.get_nel())

    def jonly():
        return direct.engine.j(D, "fp64", 1e-12, 1e-5)

    def jk():
        return direct.engine.jk(D, "fp64", 1e-12, 1e-5)

    out = {}
    for name, fn in (("xc_ms", xc), ("coulomb_only_ms", jonly), ("j_and_k_ms", jk)):
        for _ in range(max(a.warmup, 1)):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(a.steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            fn()
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        out[name] = float(np.median(ts))
    npts, nbf = gr.ng, gr.nbf
    print(json.dumps({"metric": "SVWN DFT Fock-build parts on (H2O)8", "value": out["xc_ms"] + out["coulomb_only_ms"],
                      "unit": "ms (XC + Coulomb build)", "higher_is_better": False, "steps": a.steps,
                      "data": "synthetic", "dtype": "f64",
                      "config": dict(out, workload=WORKLOAD, grid_points=npts, nbf=nbf, energy=e, scf_s=scf_s,
                                     bfgrid_bytes=8 * npts * nbf,
                                     path="pqb_grid_amps/pqb_grid_rowdot/pqb_xc_svwn + cuBLAS DGEMM; "
                                          "pqb_jk_direct with K = NULL")}))


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
        return
    if a.workload != "h2o8":
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        {"stored": run_stored, "c16h34": run_c16h34, "h2o4-grad": run_h2o4_grad,
         "batch": run_batch, "mp2": run_mp2, "dft": run_dft}[a.workload](a)
        return
    import ctypes

    import torch
    import torch.distributed as dist

    from pyquante_b200 import Ints, _lib
    from pyquante_b200.Basis.basis import BasisSet
    from pyquante_b200.LA2 import geigh, mkdens
    from pyquante_b200.engine import BasisEngine
    from pyquante_b200.flops import class_flops, quartet_class_ls

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier()

    mol = molecule()
    bs = BasisSet(mol, "6-31g**")
    n = len(bs)
    Q = nominal_quartets(n)
    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        # before any CUDA work in this process: the baseline forks workers
        cpu = reference_rate(bs, a.cpu_seconds)
    from pyquante_b200.parallel import allreduce_jk, shard_plan
    eng = BasisEngine(bs.bfs, device=local)
    counts = eng.plan(SCHWARZ, FP32_THRESH)
    shard_plan(eng, rank, world)
    qa = (ctypes.c_int64 * 42)()
    pa = (ctypes.c_int64 * 42)()
    eng.ctx.check(eng.ctx.lib.pqb_plan_stats(eng.ctx.h, qa, pa))
    qs = np.array(qa[:]).reshape(2, 21)
    ps = np.array(pa[:]).reshape(2, 21)
    kept_shell_quartets = counts["shell_quartets"] - counts["dropped"]
    prim_quartets = int(ps.sum())
    # a realistic density: a few SCF iterations from the core guess
    S, h = Ints.get1ints(bs, mol)
    St = torch.as_tensor(S, device="cuda")
    ht = torch.as_tensor(h, device="cuda")
    nocc = mol.get_nel() // 2
    _, C = geigh(ht, St)
    for _ in range(3):
        D = mkdens(C, 0, nocc).contiguous()
        J, K = eng.jk(D, "fp64", SCHWARZ, FP32_THRESH)
        allreduce_jk(J, K)
        _, C = geigh(ht + 2 * J - K, St)
    D = mkdens(C, 0, nocc).contiguous()
    if a.profile_builds:
        for _ in range(a.profile_builds):
            eng.jk(D, a.precision, SCHWARZ, FP32_THRESH)
        torch.cuda.synchronize()
        print("profile builds done")
        return
    J = torch.empty_like(D)
    K = torch.empty_like(D)
    G = torch.empty_like(D)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()

    def build(mode, e=eng):
        e.jk(D, mode, e._plan_key[0], e._plan_key[1], J=J, K=K)
        allreduce_jk(J, K)
        torch.sub(J.mul(2.0), K, out=G)

    use_graph = world == 1 and not a.no_graph
    graphs = {}

    def capture(key, fn):
        # one Fock build (memsets, class launches over the context's streams,
        # symmetrisation, G) captured once and replayed per step
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            fn()
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            fn()
        torch.cuda.synchronize()
        graphs[key] = g

    def runner(key, fn):
        return (lambda: graphs[key].replay()) if use_graph else fn

    modes = {"fp64": lambda: build("fp64"), "mixed": lambda: build("mixed")}
    for _ in range(a.warmup):
        for fn in modes.values():
            fn()
    torch.cuda.synchronize()
    if use_graph:
        for key, fn in modes.items():
            capture(key, fn)
    run = {key: runner(key, fn) for key, fn in modes.items()}
    for _ in range(a.warmup):
        for fn in run.values():
            fn()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(torch.cuda.current_device()) as clk:
        # the same builds (a fixed count, identical on every rank) for about
        # 1.5 s before the timed ones, so the clock record (nvidia-smi every
        # 0.2 s) covers the GPU under this load
        for _ in range(a.soak):
            run["fp64"]()
        torch.cuda.synchronize()
        ms = _timed(run["fp64"], a.steps, stream, flush)
        ms_mixed = _timed(run["mixed"], a.steps, stream, flush)
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
    if world > 1:
        t = torch.tensor([ms, ms_mixed], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, ms_mixed = t.tolist()

    # the mixed mode's FP64 list alone (quartets with Q_ab Q_cd >= the FP32
    # threshold): the time the mixed build cannot go below however cheap the
    # FP32 quartets become
    ms_list64 = None
    if world == 1:
        eng64 = BasisEngine(bs.bfs, device=local)
        eng64.plan(FP32_THRESH, FP32_THRESH)
        fn = lambda: build("fp64", eng64)   # noqa: E731
        for _ in range(a.warmup):
            fn()
        if use_graph:
            capture("list64", fn)
        ms_list64 = _timed(runner("list64", fn), a.steps, stream, flush)
        del eng64

    # end to end through the public API: pinned host D in, host G out
    Dh = D.cpu().pin_memory()
    Gh = torch.empty_like(Dh).pin_memory()

    def e2e(precision):
        direct = Ints.DirectInts(eng, precision, SCHWARZ, FP32_THRESH)

        def step():
            if world == 1:   # get2JmK on host arrays: one C-ABI call (D in, build, G out)
                direct.get2jmk_host(Dh, Gh)
                return
            Dd = Dh.to("cuda", non_blocking=True)
            Jd, Kd = direct.jk(Dd)
            allreduce_jk(Jd, Kd)   # each rank built its shard of the quartets
            Gh.copy_(2.0 * Jd - Kd, non_blocking=True)

        for _ in range(a.warmup):
            step()
        torch.cuda.synchronize()
        barrier()
        t = _timed(step, a.steps, stream, flush)
        if world > 1:
            tt = torch.tensor([t], device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t = float(tt[0])
        return t

    e2e_ms = e2e("fp64")
    e2e_mixed_ms = e2e("mixed")

    # UHF: two densities digesting every integral of one pass (pqb_jk_direct2)
    # against one single-density build (the library replays its own graphs)
    Db = (0.8 * D).contiguous()
    uhf_ms = uhf_single_ms = None
    if world == 1:
        for _ in range(a.warmup):
            eng.jk2(D, Db, "fp64", SCHWARZ, FP32_THRESH)
            eng.jk(D, "fp64", SCHWARZ, FP32_THRESH, J=J, K=K)
        uhf_ms = _timed(lambda: eng.jk2(D, Db, "fp64", SCHWARZ, FP32_THRESH), a.steps, stream, flush)
        uhf_single_ms = _timed(lambda: eng.jk(D, "fp64", SCHWARZ, FP32_THRESH, J=J, K=K), a.steps, stream, flush)

    # roofline: per-class FP64 timing of the direct J/K kernels
    per_class = []
    # launches of one timed FP64 build: density scaling, one kernel per class
    # (an FP64 build runs both lists of a class in one launch), then one take
    # of J and K from the graph's accumulators (without the graph: one
    # symmetrise kernel each)
    nlaunch = (2 if use_graph else 3) + sum(1 for qc in range(21) if qs[0, qc] + qs[1, qc] > 0)
    for part in (0, 1):
        for qc in range(21):
            if qs[part, qc] == 0:
                continue
            tms = []
            for _ in range(3):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                eng.ctx.check(eng.ctx.lib.pqb_jk_direct_class(eng.ctx.h, _lib.ptr(D), _lib.ptr(J), _lib.ptr(K), part,
                                                              qc, _lib.PQB_FP64, _lib.stream_ptr()))
                e1.record(stream)
                e1.synchronize()
                tms.append(e0.elapsed_time(e1))
            t_ms = sorted(tms)[1]
            fl = class_flops(qc, int(ps[part, qc]), int(qs[part, qc]))
            per_class.append(dict(part=part, cls=quartet_class_ls(qc), ms=t_ms, flops=fl,
                                  tflops=fl / (t_ms * 1e-3) / 1e12, items=int(qs[part, qc]),
                                  prims=int(ps[part, qc])))
    peak = ctypes.c_double()
    eng.ctx.check(eng.ctx.lib.pqb_fp64_peak(eng.ctx.h, 200000, ctypes.byref(peak)))
    peak_tf = peak.value / 1e12
    dom = max(per_class, key=lambda r: r["ms"])
    tot_fl = sum(r["flops"] for r in per_class)
    build_tflops = tot_fl / (ms * 1e-3) / 1e12

    # accuracy of the mixed mode: RHF on each path from the same start
    scf = None
    if rank == 0:
        e64, it64, s64 = _scf(mol, bs, "fp64")
        emx, itmx, smx = _scf(mol, bs, "mixed")
        ep, itp, sp = _scf(mol, bs, "fp64", solver="purify")
        scf = dict(e64=e64, emx=emx, it64=it64, itmx=itmx, s64=s64, smx=smx, ep=ep, itp=itp, sp=sp)
    if rank == 0:
        line = {
            "metric": "ERI quartets/s (2J-K Fock build, FP64; nominal unique (ij|kl))",
            "value": Q / (ms * 1e-3), "unit": "quartets/s", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": ms, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "precision": "fp64", "schwarz": SCHWARZ, "nominal_quartets": Q,
                       "shell_quartets": counts["shell_quartets"],
                       "computed_shell_quartets": kept_shell_quartets,
                       "computed_primitive_quartets": prim_quartets,
                       "work_items": counts["fp64"] + counts["fp32"],
                       "l2": "256 MiB buffer zeroed between timed builds", "cuda_graph": use_graph,
                       "parallelism": "quartet shards x%d + NCCL all-reduce of J,K" % world if world > 1 else "1 GPU"},
            "computed_shell_quartets_per_s": kept_shell_quartets / (ms * 1e-3),
            "computed_primitive_quartets_per_s": prim_quartets / (ms * 1e-3),
            "s_per_fock_build": ms * 1e-3,
            "e2e": {"value": Q / (e2e_ms * 1e-3), "unit": "quartets/s", "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": int(D.numel() * 8), "d2h_bytes_per_step": int(D.numel() * 8),
                    "api": ("pyquante_b200.Ints.DirectInts.get2jmk_host -> pqb_get2jmk_host (get2JmK on host "
                            "arrays: D in, build, G = 2J - K out in one call), FP64, pinned host D and G"
                            if world == 1 else
                            "pyquante_b200.Ints.DirectInts.jk on each rank's shard, NCCL all-reduce of J and K, "
                            "G = 2J - K to pinned host memory")},
            "mixed": {"precision": "mixed", "fp32_threshold": FP32_THRESH, "dtype": "f64+f32",
                      "ms_per_step": ms_mixed, "value": Q / (ms_mixed * 1e-3), "unit": "quartets/s",
                      "speedup_vs_fp64": ms / ms_mixed,
                      "fp64_list_alone_ms": ms_list64,
                      "speedup_ceiling": (ms / ms_list64) if ms_list64 else None,
                      "speedup_ceiling_note": "FP64 build time over the time of the mixed mode's FP64 list alone "
                                              "(quartets with Q_ab Q_cd >= the FP32 threshold): the bound if the "
                                              "FP32 quartets cost nothing",
                      "kept_fp64_items": counts["fp64"], "kept_fp32_items": counts["fp32"],
                      "e2e": {"value": Q / (e2e_mixed_ms * 1e-3), "unit": "quartets/s", "ms_per_step": e2e_mixed_ms}},
            "roofline": {"bound": "fp64", "achieved": build_tflops, "peak": peak_tf, "unit": "TFLOP/s",
                         "frac": build_tflops / peak_tf, "traffic": DIRECT_TRAFFIC_BYTES,
                         "traffic_note": "DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum) summed over "
                                         "the class launches of one FP64 build of this workload; the build is "
                                         "L2-resident, so the FP64 pipe, not HBM, is the roofline",
                         "kernel": "eri_thread_kernel/eri_block_kernel<class, EpiJK>: all class instantiations "
                                   "of one FP64 Fock build, launched together by pqb_jk_direct",
                         "flops_per_build": tot_fl, "flop_model": "pyquante_b200.flops (per-class counts of the "
                                                                   "kernels' FP64 operations, FMA = 2)",
                         "peak_source": "measured DFMA probe (pqb_fp64_peak) on this GPU",
                         "slowest_class_alone": "(%d%d|%d%d)" % tuple(dom["cls"]),
                         "slowest_class_alone_tflops": dom["tflops"]},
            "uhf_two_density": {"ms_per_build": uhf_ms, "single_density_ms": uhf_single_ms,
                                "cost_vs_single": (uhf_ms / uhf_single_ms) if uhf_ms else None,
                                "api": "BasisEngine.jk2 -> pqb_jk_direct2 (Ja, Ka, Jb, Kb in one pass), FP64"},
            "gpu_launches": nlaunch * a.steps,
            "clocks": clk.summary(),
        }
        if scf is not None:
            line["scf"] = {"energy_fp64": scf["e64"], "energy_mixed": scf["emx"],
                           "abs_dE_mixed_vs_fp64": abs(scf["emx"] - scf["e64"]),
                           "fock_builds_fp64": scf["it64"], "fock_builds_mixed": scf["itmx"],
                           "s_per_iteration_fp64": scf["s64"] / max(scf["it64"], 1),
                           "s_per_iteration_mixed": scf["smx"] / max(scf["itmx"], 1),
                           "convergence": "RHF, DIIS, |dE| < 1e-10 Eh, core guess; host eigensolver",
                           "device_purification": {"energy_fp64": scf["ep"], "fock_builds": scf["itp"],
                                                   "s_per_iteration": scf["sp"] / max(scf["itp"], 1),
                                                   "abs_dE_vs_eigensolver": abs(scf["ep"] - scf["e64"]),
                                                   "loop": "rhf(solver='purify'): SCF loop on the GPU, "
                                                           "densities by canonical purification"}}
            line["mixed"]["abs_dE_vs_fp64"] = line["scf"]["abs_dE_mixed_vs_fp64"]
        if cpu is not None:
            line["cpu_baseline"] = {"value": cpu["value"], "unit": "quartets/s", "cores": cpu["cores"],
                                    "kind": "reference",
                                    "sample": "%d quartets (%d random bra rows, all kl >= ij) in %.1f s" % (
                                        cpu["quartets"], cpu["rows"], cpu["seconds"])}
        line["per_class_fp64"] = [dict(cls="%d%d|%d%d" % r["cls"], part=r["part"], ms=round(r["ms"], 4),
                                       tflops=round(r["tflops"], 3), items=r["items"], prims=r["prims"])
                                  for r in sorted(per_class, key=lambda r: -r["ms"])]
        print(json.dumps(line))
    if world > 1:
        graphs.clear()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
