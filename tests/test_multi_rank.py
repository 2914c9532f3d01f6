"""World-size-2 gloo runs of the multi-GPU Fock-build protocol.

On the CPU: each rank digests its share (every 2nd unique quartet, the rule
of parallel.shard_indices) into partial J/K with the same unique-quartet
weights the kernels use; parallel.allreduce_jk sums them; the result must
equal the oracle's full J and K.

On one GPU (marked gpu): two rank processes, each with its own context on
cuda:0, shard the plan with the shipped pqb_plan_shard (parallel.sharded_jk),
build their partial J/K on the device and sum them with a gloo all-reduce of
host copies.  No kernel of one rank waits on the other; the only exchange is
the host-side collective.  The sum must equal the one-rank build."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _partial_jk(ints, D, rank, world):
    """Unique-quartet digestion (the EpiJK formulas) over this rank's items."""
    import pyq_oracle as O
    from pyquante_b200.parallel import shard_indices
    n = D.shape[0]
    quartets = [(i, j, k, l) for i in range(n) for j in range(i + 1) for k in range(n) for l in range(k + 1)
                if i * (i + 1) // 2 + j >= k * (k + 1) // 2 + l]
    Jacc = np.zeros((n, n))
    Kacc = np.zeros((n, n))
    for t in shard_indices(len(quartets), rank, world):
        i, j, k, l = quartets[t]
        v = ints[O.ijkl2intindex(i, j, k, l)]
        v *= (0.5 if i == j else 1.0) * (0.5 if k == l else 1.0)
        v *= 0.5 if (i * (i + 1) // 2 + j) == (k * (k + 1) // 2 + l) else 1.0
        Jacc[i, j] += 2 * v * D[k, l]
        Jacc[k, l] += 2 * v * D[i, j]
        Kacc[i, k] += v * D[j, l]
        Kacc[i, l] += v * D[j, k]
        Kacc[j, k] += v * D[i, l]
        Kacc[j, l] += v * D[i, k]
    return Jacc + Jacc.T, Kacc + Kacc.T


def _worker(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "oracle"))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import pyq_oracle as O
        from pyquante_b200 import geometries
        from pyquante_b200.Basis.sto3g import basis_data
        from pyquante_b200.parallel import allreduce_jk
        mol = geometries.water_cluster(2, seed=1)
        atoms = [(a.atno, tuple(a.r)) for a in mol.atoms]
        bfs = O.build_basis(atoms, basis_data)
        ints = O.orc_get2ints(bfs)
        rng = np.random.default_rng(0)
        C = rng.standard_normal((len(bfs), 5))
        D = C @ C.T
        Jp, Kp = _partial_jk(ints, D, rank, world)
        J = torch.tensor(Jp)
        K = torch.tensor(Kp)
        allreduce_jk(J, K)
        if rank == 0:
            Jo, Ko = O.getJK(ints, D)
            q.put((float(np.abs(J.numpy() - Jo).max()), float(np.abs(K.numpy() - Ko).max())))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharded_fock_build_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    ej, ek = q.get(timeout=5)
    assert ej < 1e-10 and ek < 1e-10


def _gpu_worker(rank, world, port, q):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        from pyquante_b200 import geometries
        from pyquante_b200.Basis.basis import BasisSet
        from pyquante_b200.engine import BasisEngine
        from pyquante_b200.parallel import sharded_jk
        torch.cuda.set_device(0)
        mol = geometries.water_cluster(3, seed=2)
        bs = BasisSet(mol, "6-31g**")
        n = len(bs)
        rng = np.random.default_rng(0)
        C = rng.standard_normal((n, 10)) * 0.3
        D = torch.as_tensor(C @ C.T, device="cuda")
        from pyquante_b200 import parallel
        # this rank's share of the plan (pqb_plan_shard), built on the device,
        # summed over ranks on the host
        eng = BasisEngine(bs.bfs, device=0)
        eng.plan(1e-12, 1e-5)
        parallel.shard_plan(eng, rank, world)
        Jp, Kp = eng.jk(D, "fp64", 1e-12)
        J = Jp.cpu()
        K = Kp.cpu()
        parallel.allreduce_jk(J, K)
        # the same through the helper a caller uses (plan, shard, build, all-reduce)
        Jh, Kh = sharded_jk(BasisEngine(bs.bfs, device=0), D.cpu(), "fp64", 1e-12)
        if rank == 0:
            full = BasisEngine(bs.bfs, device=0)
            Jf, Kf = full.jk(D, "fp64", 1e-12)
            Jf, Kf = Jf.cpu(), Kf.cpu()
            q.put((float((J - Jf).abs().max() / Jf.abs().max()), float((K - Kf).abs().max() / Kf.abs().max()),
                   float((Jh.cpu() - Jf).abs().max() / Jf.abs().max())))
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_two_rank_sharded_device_build_gloo():
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gpu_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    ej, ek, eh = q.get(timeout=5)
    assert ej < 1e-12 and ek < 1e-12 and eh < 1e-12


def test_shard_rule_partitions_every_item():
    from pyquante_b200.parallel import shard_indices
    for n in (0, 1, 7, 100):
        for w in (1, 2, 3, 8):
            got = sorted(i for r in range(w) for i in shard_indices(n, r, w))
            assert got == list(range(n))
