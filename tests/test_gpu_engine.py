"""GPU parity: the CUDA engine through the C ABI against the oracle, the
reference's compiled C (oracle/_ref, when present) and the golden fixtures.

Tolerances (FP64 path): 1e-10 absolute per integral, 1e-8 Eh total energy,
1e-10 on J/K elements; mixed precision: stated per test."""
import json
import os

import numpy as np
import pytest

import pyq_oracle as O
from conftest import GOLDEN

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from pyquante_b200 import Ints, _lib, chgp, cints, crys, geometries  # noqa: E402
from pyquante_b200.Basis.basis import BasisSet  # noqa: E402
from pyquante_b200.engine import BasisEngine  # noqa: E402
from pyquante_b200.hartree_fock import rhf  # noqa: E402

ERI_TOL = 1e-10
E_TOL = 1e-8


def atoms_of(mol):
    return [(a.atno, tuple(float(c) for c in a.r)) for a in mol.atoms]


def oracle_bfs(bs):
    return [O.BF(bf.origin, bf.powers, list(zip(bf.pexps, bf.pcoefs))) for bf in bs.bfs]


# ------------------------------------------------------------ Boys / Rys --
def test_boys_device_matches_40_digit_values():
    ctx = _lib.context()
    g = json.load(open(os.path.join(GOLDEN, "boys.json")))
    for m in sorted({int(r[0]) for r in g["mpmath"]}):
        rows = [r for r in g["mpmath"] if r[0] == m]
        T = torch.tensor([r[1] for r in rows], dtype=torch.float64, device="cuda")
        F = torch.empty(len(rows) * (m + 1), dtype=torch.float64, device="cuda")
        ctx.check(ctx.lib.pqb_boys_eval(ctx.h, m, len(rows), _lib.ptr(T), _lib.ptr(F), _lib.stream_ptr()))
        got = F.view(len(rows), m + 1)[:, m].cpu().numpy()
        ref = np.array([r[2] for r in rows])
        assert np.all(np.abs(got - ref) <= 2e-14 * np.abs(ref)), (m, got, ref)
    # TestMath.c:18-19 through the cints drop-in
    assert abs(cints.Fgamma(0, 1.0) - 0.7468241328124271) < 1e-8
    assert abs(cints.Fgamma(0.5, 6.8) - 0.073447516533246701) < 1e-8


def test_compact_row_boys_of_the_thread_kernels():
    """The branch-free compact-row Boys form of the thread-mode kernels
    (pqb_boys_rows_eval): F_m, m <= 4, against the 40-digit values, and
    F_0..F_4 on a dense sweep of T (both sides of the table's end at T = 40,
    where the exp(-T) estimate enters the large-T recursion) against the
    general evaluation, 2e-14 relative."""
    ctx = _lib.context()
    g = json.load(open(os.path.join(GOLDEN, "boys.json")))
    for m in (0, 1, 2, 4):
        rows = [r for r in g["mpmath"] if r[0] == m]
        T = torch.tensor([r[1] for r in rows], dtype=torch.float64, device="cuda")
        F = torch.empty(len(rows) * (m + 1), dtype=torch.float64, device="cuda")
        ctx.check(ctx.lib.pqb_boys_rows_eval(ctx.h, m, len(rows), _lib.ptr(T), _lib.ptr(F), _lib.stream_ptr()))
        got = F.view(len(rows), m + 1)[:, m].cpu().numpy()
        ref = np.array([r[2] for r in rows])
        assert np.all(np.abs(got - ref) <= 2e-14 * np.abs(ref)), (m, got, ref)
    T = torch.cat([torch.linspace(0.0, 45.0, 40001, dtype=torch.float64),
                   torch.linspace(39.9, 40.1, 2001, dtype=torch.float64),
                   torch.logspace(1.6, 6.0, 2001, dtype=torch.float64)]).cuda()
    n = T.numel()
    for lt in range(5):
        Fr = torch.empty(n * (lt + 1), dtype=torch.float64, device="cuda")
        Fg = torch.empty(n * (lt + 1), dtype=torch.float64, device="cuda")
        ctx.check(ctx.lib.pqb_boys_rows_eval(ctx.h, lt, n, _lib.ptr(T), _lib.ptr(Fr), _lib.stream_ptr()))
        ctx.check(ctx.lib.pqb_boys_eval(ctx.h, lt, n, _lib.ptr(T), _lib.ptr(Fg), _lib.stream_ptr()))
        rel = ((Fr - Fg).abs() / Fg.abs()).max().item()
        assert rel < 2e-14, (lt, rel)


def test_rys_roots_weights_match_40_digit_values():
    ctx = _lib.context()
    g = np.load(os.path.join(GOLDEN, "rys.npz"))
    T = torch.tensor(g["T"], dtype=torch.float64, device="cuda")
    for n in range(1, 6):
        u = torch.empty(len(g["T"]) * n, dtype=torch.float64, device="cuda")
        w = torch.empty_like(u)
        ctx.check(ctx.lib.pqb_rys_eval(ctx.h, n, len(g["T"]), _lib.ptr(T), _lib.ptr(u), _lib.ptr(w),
                                       _lib.stream_ptr()))
        uu = u.view(-1, n).cpu().numpy()
        ww = w.view(-1, n).cpu().numpy()
        assert np.all(np.abs(uu - g["u%d" % n]) <= 1e-14 * np.abs(g["u%d" % n]) + 1e-300), n
        assert np.all(np.abs(ww - g["w%d" % n]) <= 1e-14 * np.abs(g["w%d" % n]) + 1e-300), n


# ------------------------------------------------------- packed integrals --
def test_packed_sto3g_water_vs_reference_golden():
    mol = geometries.water()
    bs = BasisSet(mol, "sto-3g")
    ints = Ints.get2ints(bs)
    gold = np.load(os.path.join(GOLDEN, "eri_sto3g_water.npy"))
    assert len(ints) == 406
    assert np.abs(ints.numpy() - gold).max() < ERI_TOL


def test_packed_631ss_water_vs_reference_and_oracle():
    mol = geometries.water()
    bs = BasisSet(mol, "6-31g**")
    assert len(bs) == 25
    ints = Ints.get2ints(bs).numpy()
    s = np.load(os.path.join(GOLDEN, "eri_631ss_water_sample.npz"))
    assert np.abs(ints[s["index"]] - s["value"]).max() < ERI_TOL
    orc = O.orc_get2ints(oracle_bfs(bs))
    assert np.abs(ints - orc).max() < ERI_TOL


def test_packed_two_waters_every_class_vs_oracle():
    mol = geometries.water_cluster(2, seed=4)
    bs = BasisSet(mol, "6-31g**")
    ints = Ints.get2ints(bs).numpy()
    orc = O.orc_get2ints(oracle_bfs(bs))
    assert np.abs(ints - orc).max() < ERI_TOL


def test_packed_h2o8_sample_vs_reference_engine():
    """(H2O)8 / 6-31G**, N = 200, Q = 202,015,050 integrals (1.6 GB)."""
    mol = geometries.water_cluster(8, seed=0)
    bs = BasisSet(mol, "6-31g**")
    assert len(bs) == 200
    eng = BasisEngine(bs.bfs)
    t = eng.eri_packed()
    assert t.numel() == 202015050
    s = np.load(os.path.join(GOLDEN, "eri_631ss_h2o8_sample.npz"))
    idx = np.array([O.ijkl2intindex(*q) for q in s["quartets"]])
    got = t[torch.from_numpy(idx).cuda()].cpu().numpy()
    assert np.abs(got - s["value"]).max() < ERI_TOL
    # size-independent property: every slot written once, finite
    assert bool(torch.isfinite(t).all())
    del t


# --------------------------------------------------------- one-electron --
def test_one_electron_vs_oracle():
    for mol, basis in [(geometries.water(), "sto-3g"), (geometries.water_cluster(2, seed=1), "6-31g**")]:
        bs = BasisSet(mol, basis)
        S, h = Ints.get1ints(bs, mol)
        So, ho = O.orc_get1ints(oracle_bfs(bs), atoms_of(mol))
        assert np.abs(S - So).max() < 1e-12
        assert np.abs(h - ho).max() < 1e-10


# ----------------------------------------------------------- scalar API --
def test_scalar_entry_points_vs_reference():
    rng = np.random.default_rng(2)
    mol = geometries.water_cluster(2, seed=7)
    bs = BasisSet(mol, "6-31g**")
    bfs = bs.bfs
    have_ref = O.ref_available()
    for _ in range(12):
        i, j, k, l = (int(x) for x in rng.integers(0, len(bfs), 4))
        a, b, c, d = bfs[i], bfs[j], bfs[k], bfs[l]
        args = []
        for f in (a, b, c, d):
            args += [f.pexps, f.pcoefs, f.pnorms, f.origin, f.powers]
        ob = [O.BF(f.origin, f.powers, list(zip(f.pexps, f.pcoefs))) for f in (a, b, c, d)]
        want = O.orc_contr(*ob)
        if have_ref:
            assert abs(O.ref_contr(*ob) - want) < 1e-12
        assert abs(crys.contr_coulomb(*args) - want) < ERI_TOL
        assert abs(cints.contr_coulomb(*args) - want) < ERI_TOL
        assert abs(chgp.contr_coulomb(*args) - want) < ERI_TOL
        pa = (a.origin, a.pnorms[0], a.powers, a.pexps[0])
        pb = (b.origin, b.pnorms[0], b.powers, b.pexps[0])
        pc = (c.origin, c.pnorms[0], c.powers, c.pexps[0])
        pd = (d.origin, d.pnorms[0], d.powers, d.pexps[0])
        v1 = crys.coulomb_repulsion(*pa, *pb, *pc, *pd)
        v2 = chgp.coulomb_repulsion(*pa, *pb, *pc, *pd)
        assert abs(v1 - v2) <= 1e-12 * max(1.0, abs(v1))
        if have_ref:
            rc = O.ref_lib("crys")
            r = rc.coulomb_repulsion(*pa[0], pa[1], *pa[2], pa[3], *pb[0], pb[1], *pb[2], pb[3],
                                     *pc[0], pc[1], *pc[2], pc[3], *pd[0], pd[1], *pd[2], pd[3])
            assert abs(v1 - r) <= 1e-12 * max(1.0, abs(r))
            # chgp.vrr with m > 0 against the reference (its Boys is 3e-7 accurate)
            rh = O.ref_lib("chgp")
            for m in (0, 1, 2):
                want_v = rh.ref_chgp_vrr(*pa[0], pa[1], *pa[2], pa[3], *pb[0], pb[1], pb[3],
                                         *pc[0], pc[1], *pc[2], pc[3], *pd[0], pd[1], pd[3], m)
                got_v = chgp.vrr(pa[0], pa[1], pa[2], pa[3], pb[0], pb[1], pb[3], pc[0], pc[1], pc[2], pc[3],
                                 pd[0], pd[1], pd[3], m)
                assert abs(got_v - want_v) <= 1e-6 * abs(want_v) + 1e-12


def test_scalar_errors_are_raised_not_garbage():
    f = [[1.0], [1.0], [1.0], (0.0, 0.0, 0.0)]
    with pytest.raises(_lib.EngineError):   # total L = 12 > 9: the reference silently uses stale roots
        crys.contr_coulomb(*(f + [(3, 0, 0)]) * 4)
    with pytest.raises(ValueError):
        crys.contr_coulomb([1.0, 2.0], [1.0], [1.0], (0, 0, 0), (0, 0, 0), *(f + [(0, 0, 0)]) * 3)


def test_general_per_function_path_vs_oracle():
    """Functions that do not form shells (reordered list): per-function kernel."""
    mol = geometries.water()
    bs = BasisSet(mol, "6-31g**")
    rng = np.random.default_rng(0)
    order = rng.permutation(len(bs))
    bfs = [bs.bfs[i] for i in order]
    ints = Ints.get2ints(bfs)
    assert not ints.engine.has_shells
    orc = O.orc_get2ints([O.BF(f.origin, f.powers, list(zip(f.pexps, f.pcoefs))) for f in bfs])
    assert np.abs(ints.numpy() - orc).max() < ERI_TOL


# ------------------------------------------------------------------ J / K --
def _rand_density(n, seed=0):
    rng = np.random.default_rng(seed)
    C = rng.standard_normal((n, max(1, n // 3))) * 0.3
    return C @ C.T


def test_jk_stored_and_direct_vs_oracle():
    mol = geometries.water_cluster(2, seed=4)
    bs = BasisSet(mol, "6-31g**")
    D = _rand_density(len(bs))
    orc = O.orc_get2ints(oracle_bfs(bs))
    Jo, Ko = O.getJK(orc, D)
    ints = Ints.get2ints(bs)
    J, K = Ints.getJ(ints, D), Ints.getK(ints, D)
    assert np.abs(J - Jo).max() < ERI_TOL and np.abs(K - Ko).max() < ERI_TOL
    G = Ints.get2JmK(ints, D)
    assert np.abs(G - (2 * Jo - Ko)).max() < 2 * ERI_TOL
    d = Ints.get2ints(bs, direct=True, schwarz=0.0)
    Jd, Kd = Ints.getJ(d, D), Ints.getK(d, D)
    assert np.abs(Jd - Jo).max() < ERI_TOL and np.abs(Kd - Ko).max() < ERI_TOL
    # host arrays through pqb_get2jmk_host on a fresh handle: the first call
    # builds without the graph (J, K, then G), the next ones replay it and
    # take G from the accumulators
    d2 = Ints.get2ints(bs, direct=True, schwarz=0.0)
    for _ in range(3):
        Gh = Ints.get2JmK(d2, D)
        assert isinstance(Gh, np.ndarray) and np.abs(Gh - (2 * Jo - Ko)).max() < 2 * ERI_TOL
    Dp = torch.as_tensor(D).pin_memory()
    Gp = torch.empty_like(Dp).pin_memory()
    d2.get2jmk_host(Dp, Gp)
    torch.cuda.synchronize()
    assert np.abs(Gp.numpy() - (2 * Jo - Ko)).max() < 2 * ERI_TOL
    # torch in -> torch out, same values
    Dt = torch.as_tensor(D, device="cuda")
    Gt = Ints.get2JmK(d, Dt)
    assert isinstance(Gt, torch.Tensor) and Gt.is_cuda
    assert np.abs(Gt.cpu().numpy() - (2 * Jo - Ko)).max() < 2 * ERI_TOL


def test_stored_jk_kernels_agree_with_oracle_and_direct():
    """pqb_jk_packed: the register-form kernel (nbf <= 256 and 257..512
    variants) and the one-block-per-row kernel give the same J and K; small
    case against the oracle, (H2O)11 / 6-31G** (N = 275) against the direct
    FP64 build."""
    from pyquante_b200.engine import jk_packed
    mol = geometries.water_cluster(2, seed=4)
    bs = BasisSet(mol, "6-31g**")
    D = _rand_density(len(bs))
    Jo, Ko = O.getJK(O.orc_get2ints(oracle_bfs(bs)), D)
    ints = Ints.get2ints(bs).tensor
    Dt = torch.as_tensor(D, device="cuda")
    ctx = _lib.Context(torch.cuda.current_device())
    for simple in (0, 1):
        ctx.check(ctx.lib.pqb_set_param(ctx.h, _lib.PQB_PARAM_PACKED_KERNEL, 0, simple))
        J, K = jk_packed(ints, Dt, ctx)
        assert np.abs(J.cpu().numpy() - Jo).max() < ERI_TOL, simple
        assert np.abs(K.cpu().numpy() - Ko).max() < ERI_TOL, simple
    mol = geometries.water_cluster(11, seed=1, box_ang=10.1)
    bs = BasisSet(mol, "6-31g**")
    n = len(bs)
    assert 256 < n <= 512
    D = _rand_density(n, 3)
    Dt = torch.as_tensor(D, device="cuda")
    eng = BasisEngine(bs.bfs)
    Jd, Kd = eng.jk(Dt, "fp64", 0.0)
    ints = eng.eri_packed()
    ctx.check(ctx.lib.pqb_set_param(ctx.h, _lib.PQB_PARAM_PACKED_KERNEL, 0, 0))
    J, K = jk_packed(ints, Dt, ctx)
    assert float((J - Jd).abs().max()) < 1e-9 and float((K - Kd).abs().max()) < 1e-9
    del ints
    torch.cuda.empty_cache()


@pytest.mark.parametrize("n", [50, 100, 180, 210, 256, 300, 380, 420])
def test_stored_register_kernel_every_row_width(n):
    """pqb_jk_packed's register kernel is instantiated for 2, 4, 6, 7, 8, 10,
    12 and 16 column chunks of 32 (the smallest that holds N); each width, on
    seeded random packed values (any packed array is a valid 8-fold
    symmetric tensor), against the one-block-per-row kernel."""
    from pyquante_b200.engine import jk_packed
    P = n * (n + 1) // 2
    g = torch.Generator(device="cuda").manual_seed(n)
    ints = torch.rand(P * (P + 1) // 2, dtype=torch.float64, device="cuda", generator=g) - 0.5
    Dt = torch.as_tensor(_rand_density(n, n), device="cuda")
    ctx = _lib.Context(torch.cuda.current_device())
    out = []
    for simple in (1, 0):
        ctx.check(ctx.lib.pqb_set_param(ctx.h, _lib.PQB_PARAM_PACKED_KERNEL, 0, simple))
        out.append(jk_packed(ints, Dt, ctx))
    (Js, Ks), (Jr, Kr) = out
    scale = float(Dt.abs().sum())
    assert float((Jr - Js).abs().max()) < 1e-12 * scale * n
    assert float((Kr - Ks).abs().max()) < 1e-12 * scale * n
    assert torch.equal(Jr, Jr.T) and torch.equal(Kr, Kr.T)
    del ints
    torch.cuda.empty_cache()


def test_direct_build_graph_replay_matches_launches():
    """pqb_jk_direct replays a captured CUDA graph of its class launches from
    the second call per mode on; replays, one-by-one launches and a re-plan
    (which drops and recaptures the graph) give the same J and K."""
    mol = geometries.water_cluster(3, seed=2)
    bs = BasisSet(mol, "6-31g**")
    eng = BasisEngine(bs.bfs)
    D = torch.as_tensor(_rand_density(len(bs), 5), device="cuda")
    for mode in ("fp64", "mixed"):
        runs = {}
        for graph in (0, 1):
            eng.ctx.check(eng.ctx.lib.pqb_set_param(eng.ctx.h, _lib.PQB_PARAM_GRAPH, 0, graph))
            # first call launches one by one, the second captures and replays, the third replays
            runs[graph] = [tuple(x.clone() for x in eng.jk(D, mode, 1e-12, 1e-5)) for _ in range(3)]
        J0, K0 = runs[0][0]
        scale = float(J0.abs().max())
        for graph in (0, 1):
            for J, K in runs[graph]:
                assert float((J - J0).abs().max()) < 1e-13 * scale
                assert float((K - K0).abs().max()) < 1e-13 * scale
        # a different plan: the graph is rebuilt for it
        eng.ctx.check(eng.ctx.lib.pqb_set_param(eng.ctx.h, _lib.PQB_PARAM_GRAPH, 0, 1))
        Jl, Kl = eng.jk(D, mode, 1e-7, 1e-5)
        Jr, Kr = eng.jk(D, mode, 1e-7, 1e-5)
        eng.ctx.check(eng.ctx.lib.pqb_set_param(eng.ctx.h, _lib.PQB_PARAM_GRAPH, 0, 0))
        Je, Ke = eng.jk(D, mode, 1e-7, 1e-5)
        assert float((Jr - Je).abs().max()) < 1e-13 * scale and float((Kr - Ke).abs().max()) < 1e-13 * scale
        assert float((Jl - Je).abs().max()) < 1e-13 * scale
        assert float((Je - J0).abs().max()) > 0.0   # the looser plan really differs
    eng.ctx.check(eng.ctx.lib.pqb_set_param(eng.ctx.h, _lib.PQB_PARAM_GRAPH, 0, 1))


def test_plan_is_the_same_on_any_number_of_host_threads():
    """pqb_plan enumerates bra-pair ranges and orders the class lists on
    several host threads: the plan (per-class item and primitive counts) and
    J/K equal the one-thread plan's, for thread counts that split the pairs
    unevenly."""
    import ctypes
    mol = geometries.water_cluster(3, seed=2)
    bs = BasisSet(mol, "6-31g**")
    eng = BasisEngine(bs.bfs)
    D = torch.as_tensor(_rand_density(len(bs), 7), device="cuda")
    out = {}
    for threads in (1, 3, 8, 0):
        eng.ctx.check(eng.ctx.lib.pqb_set_param(eng.ctx.h, _lib.PQB_PARAM_THREADS, 0, threads))
        eng._plan_key = None
        counts = dict(eng.plan(1e-10, 1e-5))
        qa = (ctypes.c_int64 * 42)()
        pa = (ctypes.c_int64 * 42)()
        eng.ctx.check(eng.ctx.lib.pqb_plan_stats(eng.ctx.h, qa, pa))
        J, K = eng.jk(D, "mixed", 1e-10, 1e-5)
        out[threads] = (counts, list(qa), list(pa), J.clone(), K.clone())
    c1, q1, p1, J1, K1 = out[1]
    assert c1["fp64"] > 0 and c1["fp32"] > 0 and c1["dropped"] > 0
    scale = float(J1.abs().max())
    for threads in (3, 8, 0):
        c, q, p, J, K = out[threads]
        assert c == c1 and q == q1 and p == p1, threads
        assert float((J - J1).abs().max()) < 1e-13 * scale and float((K - K1).abs().max()) < 1e-13 * scale


def test_jk_mixed_precision_error_is_small():
    mol = geometries.water_cluster(3, seed=2)
    bs = BasisSet(mol, "6-31g**")
    D = _rand_density(len(bs), 1)
    e64 = Ints.get2ints(bs, direct=True, precision="fp64", schwarz=1e-12)
    emx = Ints.get2ints(bs, direct=True, precision="mixed", schwarz=1e-12, fp32_threshold=1e-5)
    G64 = Ints.get2JmK(e64, D)
    Gmx = Ints.get2JmK(emx, D)
    counts = emx.engine.plan_counts
    assert counts["fp32"] > 0
    # FP32 only where Q_ab Q_cd < 1e-5: element errors stay ~1e-5 * 1e-7 * |D| sums
    assert np.abs(G64 - Gmx).max() < 1e-8


# -------------------------------------------------------------- energies --
def test_rhf_water_sto3g_energy():
    e = json.load(open(os.path.join(GOLDEN, "energies.json")))
    mol = geometries.water()
    E, orbe, orbs = rhf(mol, basis_data="sto-3g", ConvCriteria=1e-12, MaxIter=100)
    assert abs(E - e["water_sto3g"]) < E_TOL
    E2, _, _ = rhf(mol, basis_data="sto-3g", ConvCriteria=1e-12, MaxIter=100, direct=True, schwarz=0.0)
    assert abs(E2 - e["water_sto3g"]) < E_TOL


def test_rhf_purification_solver_matches_eigensolver():
    """rhf(solver='purify'): the SCF loop on the GPU with densities by
    canonical purification gives the eigensolver loop's energy (1e-9 Eh)
    and, from its final eigensolve, the same orbital energies (1e-7)."""
    mol = geometries.water_cluster(2, seed=4)
    bs = BasisSet(mol, "6-31g**")
    kw = dict(bfs=bs, ConvCriteria=1e-10, MaxIter=80, DoAveraging=True, direct=True)
    e0, orbe0, _ = rhf(mol, **kw)
    e1, orbe1, orbs1 = rhf(mol, solver="purify", **kw)
    assert abs(e1 - e0) < 1e-9
    assert np.abs(np.asarray(orbe1) - np.asarray(orbe0)).max() < 1e-7
    assert isinstance(orbs1, np.ndarray) and orbs1.shape == (len(bs), len(bs))


def test_rhf_reference_unit_test_energies():
    """The reference's own SCF unit tests: He and Ne / 6-31G** (Tests/he.py:16
    to 1e-7, Tests/ne.py:13 to 1e-4, rhf defaults) and H2 / STO-3G, 6-31G**
    at the TestMolecules geometry (Tests/UnitSweet.py:108-126, 4 decimals).
    He also with DIIS on, which must land on the same energy."""
    from pyquante_b200.Molecule import Molecule
    he = Molecule("He", [(2, (0.0, 0.0, 0.0))])
    e, _, _ = rhf(he, ConvCriteria=1e-10, MaxIter=100)
    assert abs(e - (-2.85516040352)) < 1e-7
    e, _, _ = rhf(he, ConvCriteria=1e-10, MaxIter=100, DoAveraging=True)
    assert abs(e - (-2.85516040352)) < 1e-7
    ne = Molecule("Ne", [(10, (0.0, 0.0, 0.0))])
    e, _, _ = rhf(ne, ConvCriteria=1e-10, MaxIter=100)
    assert abs(e - (-128.474406)) < 1e-4
    h2 = Molecule("H2", [(1, (0.0, 0.0, 0.36628549)), (1, (0.0, 0.0, -0.36628549))], units="Angstrom")
    e, _, _ = rhf(h2, basis_data="sto-3g", ConvCriteria=1e-10, MaxIter=100)
    assert round(e - (-1.117099), 4) == 0
    e, _, _ = rhf(h2, basis_data="6-31g**", ConvCriteria=1e-10, MaxIter=100)
    assert round(e - (-1.131334), 4) == 0


def test_uhf_reference_no_energy(monkeypatch):
    """NO / 6-31G** UHF at 2.12955 bohr, the reference's Tests/no_uhf.py
    (-129.247769 within 1e-4, uhf defaults).  The same uhf iterations on the
    oracle's integrals (numpy J/K) must give the GPU energy to 1e-7.  Each
    iteration asks getJK2 for the reference's getJ(Da), getJ(Db), getK(Da),
    getK(Db): two stored-integral builds at most; the integral-direct UHF
    (one pass for both densities) lands on the same energy."""
    from pyquante_b200 import hartree_fock as HF
    from pyquante_b200.Molecule import Molecule
    no = Molecule("NO", atomlist=[(7, (0.0, 0.0, 0.0)), (8, (2.12955, 0.0, 0.0))], multiplicity=2)
    builds = []
    real = Ints.jk_packed

    def counted(t, D):
        builds.append(1)
        return real(t, D)

    monkeypatch.setattr(Ints, "jk_packed", counted)
    calls = []
    f = HF.getJK2
    monkeypatch.setattr(HF, "getJK2", lambda I, Da, Db: (calls.append(1), f(I, Da, Db))[1])
    e_gpu, _, _ = HF.uhf(no)
    assert abs(e_gpu - (-129.247769)) < 1e-4
    assert 0 < len(builds) <= 2 * len(calls)
    monkeypatch.setattr(HF, "getJK2", f)
    e_direct, _, _ = HF.uhf(no, direct=True, schwarz=0.0)
    assert abs(e_direct - e_gpu) < 1e-8
    # the same driver on the oracle's integrals
    bs = BasisSet(no, "6-31g**")
    obfs = oracle_bfs(bs)
    S, h = O.orc_get1ints(obfs, atoms_of(no))
    ref = O.orc_get2ints(obfs)

    def oracle_jk2(I, Da, Db):
        (Ja, Ka), (Jb, Kb) = O.getJK(I, Da), O.getJK(I, Db)
        return Ja, Jb, Ka, Kb

    monkeypatch.setattr(HF, "getJK2", oracle_jk2)
    e_orc, _, _ = HF.uhf(no, bfs=bs.bfs, integrals=(S, h, ref))
    assert abs(e_gpu - e_orc) < 1e-7


def test_two_density_build_equals_two_single_builds():
    """pqb_jk_direct2 digests every integral against both densities in one
    pass: J and K of each equal a single-density build (FP64 and mixed, on
    the launch-by-launch first call and on graph replays)."""
    mol = geometries.water_cluster(3, seed=2)
    bs = BasisSet(mol, "6-31g**")
    eng = BasisEngine(bs.bfs)
    n = len(bs)
    Da = torch.as_tensor(_rand_density(n, 11), device="cuda")
    Db = torch.as_tensor(_rand_density(n, 12) * 0.7, device="cuda")
    for mode in ("fp64", "mixed"):
        Ja, Ka = (x.clone() for x in eng.jk(Da, mode, 1e-12, 1e-5))
        Jb, Kb = (x.clone() for x in eng.jk(Db, mode, 1e-12, 1e-5))
        for _ in range(3):
            J2a, K2a, J2b, K2b = eng.jk2(Da, Db, mode, 1e-12, 1e-5)
            for got, want in ((J2a, Ja), (K2a, Ka), (J2b, Jb), (K2b, Kb)):
                assert float((got - want).abs().max()) < 1e-12 * float(want.abs().max()), mode
    # through the API: DirectInts getJK2 -> the one-pass build
    d = Ints.get2ints(bs, direct=True)
    Jda, Jdb, Kda, Kdb = Ints.getJK2(d, Da.cpu().numpy(), Db.cpu().numpy())
    Jo, Ko = eng.jk(Db, "fp64", 1e-12, 1e-5)
    assert np.abs(Jdb - Jo.cpu().numpy()).max() < ERI_TOL and np.abs(Kdb - Ko.cpu().numpy()).max() < ERI_TOL


def test_coulomb_only_build_equals_the_j_of_the_full_build():
    """pqb_jk_direct with K = NULL runs the Coulomb digestion alone: its J
    equals the full build's (FP64 and mixed, first call and graph replays);
    through the API, getJ(coulomb_only=True) then getK on the same density
    still gives the full build's K."""
    mol = geometries.water_cluster(3, seed=2)
    bs = BasisSet(mol, "6-31g**")
    eng = BasisEngine(bs.bfs)
    D = torch.as_tensor(_rand_density(len(bs), 13), device="cuda")
    for mode in ("fp64", "mixed"):
        Jf, Kf = (x.clone() for x in eng.jk(D, mode, 1e-12, 1e-5))
        for _ in range(3):
            J = eng.j(D, mode, 1e-12, 1e-5)
            assert float((J - Jf).abs().max()) < 1e-12 * float(Jf.abs().max()), mode
    d = Ints.get2ints(bs, direct=True)
    Dn = D.cpu().numpy()
    J = Ints.getJ(d, Dn, coulomb_only=True)
    K = Ints.getK(d, Dn)
    Jf, Kf = eng.jk(D, "fp64", 1e-12, 1e-5)
    assert np.abs(J - Jf.cpu().numpy()).max() < ERI_TOL and np.abs(K - Kf.cpu().numpy()).max() < ERI_TOL


def test_single_function_and_zero_density_edge_cases():
    """He / STO-3G has one function and one unique integral: packed, direct
    and stored J/K against the oracle; a zero density gives J = K = 0."""
    from pyquante_b200.Molecule import Molecule
    he = Molecule("He", [(2, (0.0, 0.0, 0.0))])
    bs = BasisSet(he, "sto-3g")
    assert len(bs) == 1
    ints = Ints.get2ints(bs)
    ref = O.orc_get2ints(oracle_bfs(bs))
    assert len(ints) == 1 and abs(ints[0] - ref[0]) < ERI_TOL
    D = np.array([[0.7]])
    Jo, Ko = O.getJK(ref, D)
    d = Ints.get2ints(bs, direct=True, schwarz=0.0)
    for src in (ints, d):
        assert abs(Ints.getJ(src, D) - Jo).max() < ERI_TOL and abs(Ints.getK(src, D) - Ko).max() < ERI_TOL
    Z = np.zeros((1, 1))
    assert np.all(Ints.get2JmK(d, Z) == 0.0) and np.all(Ints.get2JmK(ints, Z) == 0.0)
    mol = geometries.water_cluster(2, seed=4)
    d = Ints.get2ints(BasisSet(mol, "6-31g**"), direct=True)
    Z = np.zeros((50, 50))
    assert np.all(Ints.get2JmK(d, Z) == 0.0)


def test_rhf_reference_test_geometries():
    """Tests/h2o.py and Tests/h2.py known answers, and the oracle to 1e-8 Eh."""
    from pyquante_b200.Molecule import Molecule
    e = json.load(open(os.path.join(GOLDEN, "energies.json")))
    h2o = Molecule("h2o", [(8, (0.0, 0.0, 0.0)), (1, (1.0, 0.0, 0.0)), (1, (0.0, 1.0, 0.0))], units="Angstrom")
    E, _, _ = rhf(h2o, ConvCriteria=1e-12, MaxIter=100, DoAveraging=True)
    assert abs(E - e["h2o_test_literal"]) < e["h2o_test_tol"]
    assert abs(E - e["h2o_test_geometry_631ss"]) < E_TOL
    h2 = Molecule("h2", [(1, (0.0, 0.0, 0.0)), (1, (1.0, 0.0, 0.0))], units="bohr")
    E, _, _ = rhf(h2, ConvCriteria=1e-12, MaxIter=100)
    assert abs(E - e["h2_test_literal"]) < e["h2_test_tol"]
    assert abs(E - e["h2_631ss"]) < E_TOL


def test_engine_rejects_bad_shapes():
    mol = geometries.water()
    eng = BasisEngine(BasisSet(mol, "sto-3g").bfs)
    bad = torch.empty(10, dtype=torch.float64, device="cuda")
    with pytest.raises(_lib.EngineError) as ei:
        eng.ctx.check(eng.ctx.lib.pqb_eri_packed(eng.ctx.h, _lib.ptr(bad), 10, _lib.stream_ptr()))
    assert ei.value.code == _lib.PQB_E_SHAPE
    with pytest.raises(_lib.EngineError) as ei:
        eng.ctx.check(eng.ctx.lib.pqb_jk_direct(eng.ctx.h, _lib.ptr(bad), _lib.ptr(bad), _lib.ptr(bad), 0,
                                                _lib.stream_ptr()))
    assert ei.value.code == _lib.PQB_E_STATE
