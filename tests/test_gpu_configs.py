"""GPU parity at the benchmarked workloads, through the C ABI.

  * (H2O)8 / 6-31G** (N = 200): the integral-direct FP64 J/K against the
    stored-integral J/K of the packed array (itself sample-pinned to the
    reference's compiled crys at this N), the direct FP64 RHF energy against
    the packed-integral RHF energy, and the mixed-precision energy error;
  * C16H34 / 6-31G* (N = 308, Q = 1,132,237,491, a 9.06 GB packed array): a
    sample of packed integrals in the range where the reference's 32-bit
    ijkl2intindex overflows (Src/cints.c:413-425), against the reference's
    compiled crys (tests/golden/eri_631s_c16h34_sample.npz), and the FP32
    threshold sweep 1e-7 .. 1e-4 against the FP64 energy;
  * pqb_plan_shard: the partial builds of every rank add up to the full one.

Tolerances: 1e-10 on J/K elements and integrals, 1e-8 Eh between FP64
energies, 1e-6 Eh for mixed precision (the metric's own bound)."""
import os

import numpy as np
import pytest

from conftest import GOLDEN

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from pyquante_b200 import Ints, _lib, geometries  # noqa: E402
from pyquante_b200.Basis.basis import BasisSet  # noqa: E402
from pyquante_b200.LA2 import geigh, mkdens  # noqa: E402
from pyquante_b200.engine import BasisEngine, jk_packed  # noqa: E402
from pyquante_b200.hartree_fock import rhf  # noqa: E402

JK_TOL = 1e-10
E_TOL = 1e-8
MIXED_E_TOL = 1e-6
SCF = dict(ConvCriteria=1e-10, MaxIter=80, DoAveraging=True)


@pytest.fixture(scope="module")
def h2o8():
    mol = geometries.water_cluster(8, seed=0)
    bs = BasisSet(mol, "6-31g**")
    assert len(bs) == 200
    return mol, bs


def _scf_density(mol, eng, iters=3):
    """A physical density: a few SCF iterations from the core guess."""
    S, h = Ints.get1ints(eng.bfs, mol)
    St = torch.as_tensor(S, device="cuda")
    ht = torch.as_tensor(h, device="cuda")
    nocc = mol.get_nel() // 2
    _, C = geigh(ht, St)
    for _ in range(iters):
        D = mkdens(C, 0, nocc).contiguous()
        J, K = eng.jk(D, "fp64", 1e-12)
        _, C = geigh(ht + 2 * J - K, St)
    return mkdens(C, 0, nocc).contiguous()


def test_h2o8_direct_fp64_jk_equals_stored_jk(h2o8):
    mol, bs = h2o8
    eng = BasisEngine(bs.bfs)
    D = _scf_density(mol, eng)
    ints = eng.eri_packed()
    assert ints.numel() == 202015050
    Js, Ks = jk_packed(ints, D, eng.ctx)
    del ints
    torch.cuda.empty_cache()
    # unscreened: the same integrals, digested by the fused kernels
    Jd, Kd = eng.jk(D, "fp64", 0.0)
    ej, ek = float((Jd - Js).abs().max()), float((Kd - Ks).abs().max())
    print("N=200 unscreened direct vs stored: |dJ| %.3e |dK| %.3e" % (ej, ek))
    assert ej < JK_TOL and ek < JK_TOL
    # the benchmarked plan (Schwarz 1e-12): every dropped shell quartet has
    # |(ab|cd)| <= Q_ab Q_cd < 1e-12, so the screening error of an element
    # is far below the parity bound for a physical density
    Jd, Kd = eng.jk(D, "fp64", 1e-12)
    ej, ek = float((Jd - Js).abs().max()), float((Kd - Ks).abs().max())
    print("N=200 Schwarz 1e-12 direct vs stored: |dJ| %.3e |dK| %.3e" % (ej, ek))
    assert ej < JK_TOL and ek < JK_TOL


def test_h2o8_rhf_direct_fp64_and_mixed_vs_stored(h2o8):
    mol, bs = h2o8
    e_stored, _, _ = rhf(mol, bfs=bs, **SCF)
    e64, _, _ = rhf(mol, bfs=bs, direct=True, precision="fp64", schwarz=1e-12, **SCF)
    emx, _, _ = rhf(mol, bfs=bs, direct=True, precision="mixed", schwarz=1e-12, fp32_threshold=1e-5, **SCF)
    print("(H2O)8 RHF: stored %.10f direct fp64 %.10f mixed %.10f |dE| mixed-fp64 %.3e" %
          (e_stored, e64, emx, abs(emx - e64)))
    assert abs(e64 - e_stored) < E_TOL
    assert abs(emx - e64) < MIXED_E_TOL


@pytest.fixture(scope="module")
def c16h34():
    mol = geometries.alkane(16)
    bs = BasisSet(mol, "6-31g*")
    assert len(bs) == 308
    return mol, bs


def test_c16h34_packed_sample_vs_reference_engine(c16h34):
    """The 9.06 GB packed array at N = 308: the reference's 32-bit index
    overflows for ij >= 46341; this one does not."""
    mol, bs = c16h34
    eng = BasisEngine(bs.bfs)
    s = np.load(os.path.join(GOLDEN, "eri_631s_c16h34_sample.npz"))
    idx = np.array([Ints.ijkl2intindex(*(int(x) for x in q)) for q in s["quartets"]], dtype=np.int64)
    assert np.array_equal(idx, s["index"])
    P = 308 * 309 // 2
    assert int(idx.max()) >= 46341 * 46342 // 2 and idx.max() < P * (P + 1) // 2
    t = eng.eri_packed()
    assert t.numel() == P * (P + 1) // 2 == 1132237491
    got = t[torch.from_numpy(idx).cuda()].cpu().numpy()
    err = float(np.abs(got - s["value"]).max())
    print("C16H34 packed sample (%d quartets, %d in the overflow range): max |err| %.3e" %
          (len(idx), int((idx >= 46341 * 46342 // 2).sum()), err))
    assert err < JK_TOL
    assert bool(torch.isfinite(t).all())
    del t
    torch.cuda.empty_cache()


def test_c16h34_mixed_threshold_sweep(c16h34):
    mol, bs = c16h34
    e64, _, _ = rhf(mol, bfs=bs, direct=True, precision="fp64", schwarz=1e-12, **SCF)
    for thr in (1e-7, 1e-6, 1e-5, 1e-4):
        emx, _, _ = rhf(mol, bfs=bs, direct=True, precision="mixed", schwarz=1e-12, fp32_threshold=thr, **SCF)
        print("C16H34 FP32 threshold %.0e: |dE| vs FP64 %.3e Eh" % (thr, abs(emx - e64)))
        assert abs(emx - e64) < MIXED_E_TOL, thr


@pytest.mark.parametrize("nranks", [2, 3])
def test_plan_shard_partial_builds_add_up(h2o8, nranks):
    """pqb_plan_shard(rank, nranks) keeps every nranks-th work item of each
    class list; the rank builds add up to the unsharded J and K."""
    mol, bs = h2o8
    eng = BasisEngine(bs.bfs)
    D = _scf_density(mol, eng, iters=1)
    J, K = (x.clone() for x in eng.jk(D, "fp64", 1e-12))
    Js = torch.zeros_like(J)
    Ks = torch.zeros_like(K)
    items = 0
    for r in range(nranks):
        eng._plan_key = None
        full = eng.plan(1e-12, 1e-5)
        eng.ctx.check(eng.ctx.lib.pqb_plan_shard(eng.ctx.h, r, nranks))
        import ctypes
        qa = (ctypes.c_int64 * 42)()
        pa = (ctypes.c_int64 * 42)()
        eng.ctx.check(eng.ctx.lib.pqb_plan_stats(eng.ctx.h, qa, pa))
        items += sum(qa)
        Jr, Kr = eng.jk(D, "fp64", 1e-12)
        Js += Jr
        Ks += Kr
    assert items == full["fp64"] + full["fp32"]
    scale = float(J.abs().max())
    assert float((Js - J).abs().max()) < 1e-12 * scale
    assert float((Ks - K).abs().max()) < 1e-12 * float(K.abs().max())
    with pytest.raises(_lib.EngineError):
        eng.ctx.check(eng.ctx.lib.pqb_plan_shard(eng.ctx.h, nranks, nranks))
