"""GPU parity of the AO -> MO transformation and MP2 (PyQuante/MP.py:20-97)
through the C ABI gather kernels and FP64 GEMMs, against the oracle's
restatement (oracle/pyq_oracle.py: the reference's loops and a dense numpy
transform) and the reference's own MP2 known answers.

Tolerances: 1e-10 on MO integrals and MP2 energies against the oracle on
the same orbitals; the reference's test tolerances on total energies."""
import numpy as np
import pytest

import pyq_oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from pyquante_b200 import MP, Ints, geometries  # noqa: E402
from pyquante_b200.Basis.basis import BasisSet  # noqa: E402
from pyquante_b200.hartree_fock import rhf  # noqa: E402
from pyquante_b200.Molecule import Molecule  # noqa: E402

TOL = 1e-10
SCF = dict(ConvCriteria=1e-12, MaxIter=200, DoAveraging=True)


def oracle_bfs(bs):
    return [O.BF(bf.origin, bf.powers, list(zip(bf.pexps, bf.pcoefs))) for bf in bs.bfs]


def _scf(mol, basis):
    bs = BasisSet(mol, basis)
    S, h, ints = Ints.getints(bs, mol)
    e, orbe, orbs = rhf(mol, bfs=bs, integrals=(S, h, ints), **SCF)
    return bs, ints, e, orbe, orbs


def test_transform_packed_mo_integrals_vs_reference_loops():
    """Water / STO-3G: every slot of the packed MO array equals the
    step-by-step TransformIntsMP2 of the reference on the same orbitals."""
    mol = geometries.water()
    bs, ints, _, orbe, orbs = _scf(mol, "sto-3g")
    mo = MP.TransformIntsMP2(ints, orbs, 5)
    ref = O.transform_ints_mp2_loops(ints.numpy(), orbs, 5)
    assert len(mo) == len(ref)
    assert np.abs(mo.numpy() - ref).max() < TOL


def test_transform_and_mp2_vs_dense_oracle_two_waters():
    """(H2O)2 / 6-31G** (N = 50): MO integrals (ai|bj) and the MP2 energy
    against the dense numpy transform of the oracle's integrals, on the GPU
    SCF's orbitals."""
    mol = geometries.water_cluster(2, seed=4)
    bs, ints, _, orbe, orbs = _scf(mol, "6-31g**")
    n, nocc = len(bs), mol.get_nel() // 2
    orc = O.orc_get2ints(oracle_bfs(bs))
    Z = O.transform_ovov(orc, orbs, nocc)
    mo = MP.TransformIntsMP2(ints, orbs, nocc).numpy()
    k = np.array([O.ijkl2intindex(a, i, b, j) for a in range(nocc) for i in range(0, n, 7) for b in range(nocc)
                  for j in range(0, n, 5)])
    want = np.array([Z[a, i, b, j] for a in range(nocc) for i in range(0, n, 7) for b in range(nocc)
                     for j in range(0, n, 5)])
    assert np.abs(mo[k] - want).max() < TOL
    emp2 = MP.MP2(ints, orbs, orbe, nocc, n - nocc)
    eo = O.mp2(orc, orbs, orbe, nocc, n - nocc)
    print("(H2O)2 MP2 %.12f oracle %.12f" % (emp2, eo))
    assert abs(emp2 - eo) < TOL


def test_mp2_reference_test_energies():
    """The reference's MP2 tests: Tests/h2_mp2.py (1e-6), Tests/he_mp2.py
    (1e-4), Tests/lih_mp2.py and Tests/ch4_mp2.py (GAMESS-UK total and
    correction, 1e-7), all 6-31G**."""
    a2b = 1 / 0.529177249
    cases = [
        (Molecule("h2", [(1, (1.0, 0.0, 0.0)), (1, (-1.0, 0.0, 0.0))]), -1.11591861694, 1e-6, None),
        (Molecule("He", [(2, (0.0, 0.0, 0.0))]), -2.880637, 1e-4, None),
        (Molecule("lih", [(3, (0.0, 0.0, 0.0)), (1, (0.0, 0.0, 1.629912 * a2b))]), -8.0021911, 1e-6, None),
        (Molecule("ch4", [(6, (0, 0, 0)), (1, (0, 0, 1.0836058890)), (1, (1.0216334297, 0, -.3612019630)),
                          (1, (-.5108167148, .8847605034, -.3612019630)),
                          (1, (-.5108167148, -.8847605034, -.3612019630))], units="Angstrom"),
         -40.36985496, 1e-7, -0.16815019),
    ]
    for mol, ref, tol, corr in cases:
        bs, ints, e, orbe, orbs = _scf(mol, "6-31g**")
        nocc = mol.get_nel() // 2
        emp2 = MP.MP2(ints, orbs, orbe, nocc, len(bs) - nocc)
        assert abs(e + emp2 - ref) < tol, (mol.name, e + emp2, ref)
        if corr is not None:
            assert abs(emp2 - corr) < 1e-7


def test_mp2_h2o8_properties():
    """(H2O)8 / 6-31G** (N = 200, 1.6 GB of packed AO integrals, 40 occupied
    orbitals): the correlation energy is negative and does not depend on
    the batching of the first half-transformation."""
    mol = geometries.water_cluster(8, seed=0)
    bs, ints, e, orbe, orbs = _scf(mol, "6-31g**")
    nocc = mol.get_nel() // 2
    e1 = MP.MP2(ints, orbs, orbe, nocc, len(bs) - nocc)
    saved = MP._ROW_BATCH_BYTES
    try:
        MP._ROW_BATCH_BYTES = 37 << 20
        e2 = MP.MP2(ints, orbs, orbe, nocc, len(bs) - nocc)
    finally:
        MP._ROW_BATCH_BYTES = saved
    print("(H2O)8 RHF %.10f MP2 correction %.10f" % (e, e1))
    assert e1 < 0.0 and abs(e1 - e2) < 1e-11
