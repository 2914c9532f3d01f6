"""Batched SCF: many molecules in one device basis.  The batched J/K of
every block must equal each molecule's own J/K (1e-10), and the batched
SCF energies the single-molecule ones."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from pyquante_b200 import geometries  # noqa: E402
from pyquante_b200.Basis.basis import BasisSet  # noqa: E402
from pyquante_b200.batch import BatchEngine, batched_rhf  # noqa: E402
from pyquante_b200.engine import BasisEngine  # noqa: E402
from pyquante_b200.hartree_fock import rhf  # noqa: E402


def _systems():
    return [(geometries.water_cluster(k, seed=10 + k), b)
            for k, b in [(1, "sto-3g"), (2, "6-31g*"), (3, "sto-3g"), (1, "6-31g*"), (2, "6-31g**")]]


def test_batched_jk_blocks_equal_single_molecule_jk():
    systems = _systems()
    beng = BatchEngine(systems)
    beng.plan(schwarz=0.0, fp32_threshold=0.0)
    rng = np.random.default_rng(0)
    Ds = []
    for n in beng.n:
        C = rng.standard_normal((n, max(1, n // 3))) * 0.3
        Ds.append(C @ C.T)
    Dflat = torch.tensor(np.concatenate([d.reshape(-1) for d in Ds]), dtype=torch.float64, device="cuda")
    assert Dflat.numel() == beng.dense_len
    J = torch.zeros_like(Dflat)
    K = torch.zeros_like(Dflat)
    beng.jk(Dflat, J, K, "fp64")
    for b, ((mol, basis), n, off) in enumerate(zip(systems, beng.n, beng.block_off)):
        e = BasisEngine(BasisSet(mol, basis).bfs)
        Js, Ks = e.jk(torch.as_tensor(Ds[b], device="cuda"), "fp64", schwarz=0.0)
        Jb = J[off:off + n * n].view(n, n)
        Kb = K[off:off + n * n].view(n, n)
        assert float((Jb - Js).abs().max()) < 1e-10
        assert float((Kb - Ks).abs().max()) < 1e-10


def test_purification_equals_eigenprojector():
    """LA2.purify (two GEMMs and pqb_purify_step per step) gives the
    projector on the nocc lowest eigenstates, batched, with padded
    dimensions held empty; the fixed-step form (no host checks) agrees."""
    from pyquante_b200.LA2 import purify
    rng = np.random.default_rng(3)
    B, n = 6, 40
    nocc = np.array([3, 7, 10, 12, 15, 20])
    nreal = np.array([40, 40, 33, 25, 40, 31])
    F = np.zeros((B, n, n))
    for b in range(B):
        m = nreal[b]
        Q, _ = np.linalg.qr(rng.standard_normal((m, m)))
        e = np.sort(rng.uniform(-5, 5, m))
        e[nocc[b]:] += 0.5          # a gap at the Fermi level
        F[b, :m, :m] = (Q * e) @ Q.T
    pad = torch.tensor(np.arange(n)[None, :] >= nreal[:, None], device="cuda")
    Ft = torch.tensor(F, device="cuda")
    for kw in (dict(), dict(fixed=True, maxit=60)):
        P = purify(Ft, torch.tensor(nocc, dtype=torch.float64), pad=pad, **kw).cpu().numpy()
        for b in range(B):
            m = nreal[b]
            w, V = np.linalg.eigh(F[b, :m, :m])
            ref = V[:, :nocc[b]] @ V[:, :nocc[b]].T
            assert np.abs(P[b, :m, :m] - ref).max() < 1e-10, (kw, b)
            if m < n:
                assert np.abs(P[b, m:, :]).max() < 1e-12 and np.abs(P[b, :, m:]).max() < 1e-12


def test_molecule_mask_skips_masked_molecules():
    """pqb_set_molecule_mask: the masked molecules' J and K blocks come out
    zero and the others' equal the unmasked build (FP64 and mixed, with the
    mask changed between builds and cleared again)."""
    systems = _systems()
    beng = BatchEngine(systems)
    beng.plan(schwarz=1e-12, fp32_threshold=1e-5)
    rng = np.random.default_rng(1)
    Ds = []
    for n in beng.n:
        C = rng.standard_normal((n, max(1, n // 3))) * 0.3
        Ds.append(C @ C.T)
    Dflat = torch.tensor(np.concatenate([d.reshape(-1) for d in Ds]), dtype=torch.float64, device="cuda")
    for mode in ("fp64", "mixed"):
        J0, K0 = torch.zeros_like(Dflat), torch.zeros_like(Dflat)
        beng.jk(Dflat, J0, K0, mode)
        for keep in ([1, 0, 1, 0, 1], [0, 1, 0, 1, 1], [0, 0, 0, 0, 0]):
            mask = torch.tensor(keep, dtype=torch.int32, device="cuda")
            beng.set_mask(mask)
            J, K = torch.zeros_like(Dflat), torch.zeros_like(Dflat)
            beng.jk(Dflat, J, K, mode)
            for b, (n, off) in enumerate(zip(beng.n, beng.block_off)):
                sl = slice(int(off), int(off) + n * n)
                if keep[b]:
                    assert float((J[sl] - J0[sl]).abs().max()) < 1e-12 * float(J0[sl].abs().max())
                    assert float((K[sl] - K0[sl]).abs().max()) < 1e-12 * float(K0[sl].abs().max())
                else:
                    assert float(J[sl].abs().max()) == 0.0 and float(K[sl].abs().max()) == 0.0
        beng.set_mask(None)
        J, K = torch.zeros_like(Dflat), torch.zeros_like(Dflat)
        beng.jk(Dflat, J, K, mode)
        # (the same sums; the FP64 atomics add them in another order)
        assert float((J - J0).abs().max()) < 1e-12 * float(J0.abs().max())
        assert float((K - K0).abs().max()) < 1e-12 * float(K0.abs().max())


def test_density_screen_skips_small_density_items():
    """pqb_set_density_screen / pqb_shell_dmax: with the shell bounds of
    the density itself and a threshold far below every bound the build is
    the unscreened one (1e-12); with a threshold above every Q_ab Q_cd dmax
    every item is skipped (J = K = 0); a threshold in between changes J and
    K by less than the skipped items' bound allows."""
    from pyquante_b200 import _lib
    systems = _systems()
    beng = BatchEngine(systems)
    beng.plan(schwarz=1e-12, fp32_threshold=0.0)
    rng = np.random.default_rng(2)
    Ds = []
    for n in beng.n:
        C = rng.standard_normal((n, max(1, n // 3))) * 0.3
        Ds.append(C @ C.T)
    Dflat = torch.tensor(np.concatenate([d.reshape(-1) for d in Ds]), dtype=torch.float64, device="cuda")
    J0, K0 = torch.zeros_like(Dflat), torch.zeros_like(Dflat)
    beng.jk(Dflat, J0, K0, "fp64")
    dsh = torch.zeros(beng.nshell, dtype=torch.float64, device="cuda")
    lib, h = beng.ctx.lib, beng.ctx.h
    beng.ctx.check(lib.pqb_shell_dmax(h, _lib.ptr(Dflat), _lib.ptr(dsh), _lib.stream_ptr()))
    assert float(dsh.min()) > 0.0 and abs(float(dsh.max()) - float(Dflat.abs().max())) < 1e-15
    for tau, kind in ((1e-30, "none"), (1e30, "all"), (1e-6, "some")):
        beng.ctx.check(lib.pqb_set_density_screen(h, _lib.ptr(dsh), tau))
        J, K = torch.zeros_like(Dflat), torch.zeros_like(Dflat)
        beng.jk(Dflat, J, K, "fp64")
        dj, dk = float((J - J0).abs().max()), float((K - K0).abs().max())
        if kind == "none":
            assert dj < 1e-12 * float(J0.abs().max()) and dk < 1e-12 * float(K0.abs().max())
        elif kind == "all":
            assert float(J.abs().max()) == 0.0 and float(K.abs().max()) == 0.0
        else:
            assert 0.0 < max(dj, dk) < 1e-2
    beng.ctx.check(lib.pqb_set_density_screen(h, None, 0.0))
    J, K = torch.zeros_like(Dflat), torch.zeros_like(Dflat)
    beng.jk(Dflat, J, K, "fp64")
    assert float((J - J0).abs().max()) < 1e-12 * float(J0.abs().max())


@pytest.mark.parametrize("graph,solver", [(True, "purify"), (False, "purify"), (True, "eigh")])
def test_batched_rhf_matches_single_solves(graph, solver):
    """Densities by batched canonical purification (no eigensolver) or by
    diagonalisation, with and without the captured Fock build."""
    systems = _systems()
    res = batched_rhf(systems, precision="fp64", conv=1e-10, maxiter=80, graph=graph, solver=solver)
    assert res["converged"].all()
    for (mol, basis), e in zip(systems, res["energies"]):
        es, _, _ = rhf(mol, basis_data=basis, ConvCriteria=1e-10, MaxIter=100, DoAveraging=True)
        assert abs(es - e) < 1e-8, (basis, es, e)


def test_incremental_fock_builds_match_full_builds():
    """The incremental builds (density changes, screened by shell bounds of
    the change, full rebuild every 8 iterations) give the energies of full
    builds every iteration (1e-9 Eh), in FP64 and in mixed precision."""
    systems = _systems()
    for prec in ("fp64", "mixed"):
        inc = batched_rhf(systems, precision=prec, conv=1e-10, maxiter=80, incremental=True)
        full = batched_rhf(systems, precision=prec, conv=1e-10, maxiter=80, incremental=False)
        assert inc["incremental"] and not full["incremental"]
        assert inc["converged"].all() and full["converged"].all()
        assert np.abs(inc["energies"] - full["energies"]).max() < 1e-9, prec


def test_batched_rhf_64_mixed_size_systems():
    """The batched-SCF workload's recipe on 64 systems (water clusters of
    1..12 molecules, STO-3G or 6-31G*, 7..228 functions): every batched
    energy equals its single solve to 1e-8 Eh (both converged to 1e-10)."""
    systems = geometries.cluster_batch(64, seed=3)
    res = batched_rhf(systems, precision="fp64", conv=1e-10, maxiter=100, graph=True)
    assert res["converged"].all()
    worst = 0.0
    for (mol, basis), e in zip(systems, res["energies"]):
        es, _, _ = rhf(mol, basis_data=basis, ConvCriteria=1e-10, MaxIter=100, DoAveraging=True, direct=True)
        worst = max(worst, abs(es - e))
    print("64 systems: max |E_batched - E_single| %.3e, batched SCF %.2f s, p50 per molecule %.3f s" %
          (worst, res["scf_seconds"], float(np.percentile(res["scf_times"], 50))))
    assert worst < 1e-8
