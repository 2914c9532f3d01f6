"""Analytic RHF gradients (adjoint kernels) against central finite
differences of the GPU energy and of the oracle energy.

Tolerance: 1e-6 Eh/bohr (central differences, step 1e-4 bohr, SCF
converged to 1e-11 Eh)."""
import numpy as np
import pytest

import pyq_oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from pyquante_b200 import geometries  # noqa: E402
from pyquante_b200.Basis.sto3g import basis_data as STO3G  # noqa: E402
from pyquante_b200.Molecule import Molecule  # noqa: E402
from pyquante_b200.force import rhf_energy, rhf_with_gradient  # noqa: E402
from pyquante_b200.hartree_fock import rhf  # noqa: E402

H = 1e-4
TOL = 1e-6
OPTS = dict(ConvCriteria=1e-11, MaxIter=200, DoAveraging=True)


def _moved(mol, a, x, d):
    atoms = [(at.atno, tuple(at.r)) for at in mol.atoms]
    r = list(atoms[a][1])
    r[x] += d
    atoms[a] = (atoms[a][0], tuple(r))
    return Molecule("m", atoms, units="bohr")


def _fd(mol, basis):
    g = np.zeros((len(mol.atoms), 3))
    for a in range(len(mol.atoms)):
        for x in range(3):
            ep, _, _ = rhf(_moved(mol, a, x, H), basis_data=basis, **OPTS)
            em, _, _ = rhf(_moved(mol, a, x, -H), basis_data=basis, **OPTS)
            g[a, x] = (ep - em) / (2 * H)
    return g


def test_gradient_water_sto3g_vs_gpu_and_oracle_fd():
    mol = geometries.perturbed(geometries.water(), 0.05, seed=1)
    e, g, _, _ = rhf_with_gradient(mol, "sto-3g", **OPTS)
    fd = _fd(mol, "sto-3g")
    assert np.abs(g - fd).max() < TOL, (g, fd)
    assert np.abs(g.sum(axis=0)).max() < 1e-8          # translational invariance
    # oracle energy (CPU HGP restatement) finite differences
    atoms = [(a.atno, tuple(a.r)) for a in mol.atoms]

    def eo(at):
        bfs = O.build_basis(at, STO3G)
        S, h = O.orc_get1ints(bfs, at)
        return O.rhf(at, S, h, O.orc_get2ints(bfs), 5, conv=1e-12, maxiter=200, diis=True)[0]

    for a, x in [(0, 0), (1, 2), (2, 1)]:
        p = [list(r) for _, r in atoms]
        p[a][x] += H
        ep = eo([(z, tuple(r)) for (z, _), r in zip(atoms, p)])
        p[a][x] -= 2 * H
        em = eo([(z, tuple(r)) for (z, _), r in zip(atoms, p)])
        assert abs(g[a, x] - (ep - em) / (2 * H)) < TOL


def test_gradient_water_dimer_631gs_fp64_and_mixed():
    mol = geometries.perturbed(geometries.water_cluster(2, seed=3), 0.05, seed=2)
    e, g, _, _ = rhf_with_gradient(mol, "6-31g*", **OPTS)
    fd = _fd(mol, "6-31g*")
    assert np.abs(g - fd).max() < TOL
    em, gm, _, _ = rhf_with_gradient(mol, "6-31g*", precision="mixed", **OPTS)
    assert abs(em - e) < 1e-6
    assert np.abs(gm - g).max() < 1e-5


def test_autograd_function_backward_runs_the_adjoint_kernels():
    mol = geometries.perturbed(geometries.water(), 0.05, seed=4)
    R = torch.tensor(np.array([a.r for a in mol.atoms]), dtype=torch.float64, requires_grad=True)
    E = rhf_energy(R, [a.atno for a in mol.atoms], "sto-3g", **OPTS)
    (gR,) = torch.autograd.grad(E, R)
    _, g, _, _ = rhf_with_gradient(mol, "sto-3g", **OPTS)
    assert np.abs(gR.numpy() - g).max() < 1e-9


def test_gradient_h2o4_631gs_config():
    """(H2O)4 from the cluster generator, 6-31G* (76 functions), coordinates
    perturbed uniformly by +-0.05 bohr (seed 7): analytic vs central
    differences, FP64 and mixed precision, 1e-6 Eh/bohr."""
    mol = geometries.perturbed(geometries.water_cluster(4, seed=0), 0.05, seed=7)
    e, g, _, _ = rhf_with_gradient(mol, "6-31g*", **OPTS)
    fd = _fd(mol, "6-31g*")
    assert np.abs(g - fd).max() < TOL
    em, gm, _, _ = rhf_with_gradient(mol, "6-31g*", precision="mixed", **OPTS)
    assert np.abs(gm - fd).max() < TOL


@pytest.mark.parametrize("basis", ["sto-3g", "6-31g*"])
def test_adjoint_kernels_vs_restated_reference_gradient(basis):
    """pqb_grad_2e + pqb_grad_1e against the oracle's restatement of the
    reference's analytic gradient (PyQuante/force.py:48-70,
    AnalyticDerivatives.py): the same D and W (the oracle's converged RHF) go
    into both, so only the integral arithmetic differs."""
    from pyquante_b200.Basis.basis import BasisSet
    from pyquante_b200.Basis.Tools import get_basis_data
    from pyquante_b200.force import rhf_gradient_from_density
    mol = geometries.perturbed(geometries.water(), 0.05, seed=1)
    atoms = [(a.atno, tuple(a.r)) for a in mol.atoms]
    data = get_basis_data(basis)
    bfs = O.build_basis(atoms, data)
    S, h = O.orc_get1ints(bfs, atoms)
    _, orbe, orbs = O.rhf(atoms, S, h, O.orc_get2ints(bfs), 5, conv=1e-13, maxiter=300, diis=True)
    C = orbs[:, :5]
    D = C @ C.T
    W = C @ np.diag(orbe[:5]) @ C.T
    go = O.rhf_gradient(atoms, data, D, W)
    bs = BasisSet(mol, basis)
    eng = bs._pqb_engine if hasattr(bs, "_pqb_engine") else None
    if eng is None:
        from pyquante_b200.engine import BasisEngine
        eng = BasisEngine(bs.bfs)
    g = rhf_gradient_from_density(mol, eng, D, W, "fp64", 0.0)
    assert np.abs(g - go).max() < 1e-9, np.abs(g - go).max()
