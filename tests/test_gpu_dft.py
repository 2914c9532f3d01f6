"""GPU parity of the DFT path (PyQuante/dft.py, MG2 grids, SVWN) through the
C ABI grid kernels, against the oracle's restatement (oracle/pyq_oracle.py:
dft_grid, bf_amps, svwn, dft) and the reference's own DFT known answers.

Tolerances: 1e-12 on grid weights, amplitudes and functional values,
1e-8 Eh between the GPU and the oracle's energies on the same integrals'
definition, and the reference's test tolerances on its answers."""
import numpy as np
import pytest

import pyq_oracle as O

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from pyquante_b200 import Ints, geometries  # noqa: E402
from pyquante_b200.Basis.basis import BasisSet  # noqa: E402
from pyquante_b200.DFunctionals import XC  # noqa: E402
from pyquante_b200.dft import dft  # noqa: E402
from pyquante_b200.MolecularGrid import MolecularGrid  # noqa: E402
from pyquante_b200.Molecule import Molecule  # noqa: E402

A2B = 1 / 0.5291772


def atoms_of(mol):
    return [(a.atno, tuple(float(c) for c in a.r)) for a in mol.atoms]


def oracle_bfs(bs):
    return [O.BF(bf.origin, bf.powers, list(zip(bf.pexps, bf.pcoefs))) for bf in bs.bfs]


def h2o():
    return Molecule("h2o", atomlist=[(8, (0, 0, 0)), (1, (A2B, 0, 0)), (1, (0, A2B, 0))])


def test_grid_weights_and_amplitudes_vs_oracle():
    """Becke-partitioned weights of the default grid (32 x 194 points per
    atom) and the basis amplitudes on it, H2O / 6-31G**."""
    mol = h2o()
    gr = MolecularGrid(mol)
    ref = O.dft_grid(atoms_of(mol))
    assert gr.ng == len(ref) == 3 * 32 * 194
    got = gr.xyzw.cpu().numpy()
    assert np.abs(got[:, :3] - ref[:, :3]).max() < 1e-12
    assert np.abs(got[:, 3] - ref[:, 3]).max() < 1e-12 * np.abs(ref[:, 3]).max()
    bs = BasisSet(mol, "6-31g**")
    gr.set_bf_amps(bs.bfs)
    B = O.bf_amps(oracle_bfs(bs), ref)
    assert np.abs(gr.bfgrid.cpu().numpy() - B).max() < 1e-12 * np.abs(B).max()


def test_svwn_pointwise_vs_oracle():
    """S + VWN energy density and potentials, closed and open shell,
    including densities below the cutoffs."""
    rng = np.random.default_rng(5)
    ra = np.concatenate([10 ** rng.uniform(-12, 2, 400), [0.0, 1e-11, 1e-9]])
    rb = np.concatenate([ra[:200], 10 ** rng.uniform(-12, 2, 200), [0.0, 0.0, 1e-9]])
    dens = torch.as_tensor(np.stack([ra, rb]), device="cuda")
    f, va, vb, _, _, _ = XC(dens, None, functional="SVWN")
    fo, vao, vbo = O.svwn(ra, rb)
    for got, want in ((f, fo), (va, vao), (vb, vbo)):
        got = got.cpu().numpy()
        assert np.all(np.abs(got - want) <= 1e-12 * np.maximum(np.abs(want), 1e-300) + 1e-300)


def test_dft_he_reference_answer():
    """Tests/he_dft.py: He / 6-31G**, SVWN, -2.8266976 within 1e-6."""
    e, _, _ = dft(Molecule("He", atomlist=[(2, (0, 0, 0))]), ConvCriteria=1e-10, MaxIter=60)
    assert abs(e - (-2.8266976)) < 1e-6


def test_dft_h2o_vs_oracle_stored_and_direct():
    """H2O / 6-31G** SVWN (the geometry of Tests/h2o_dft.py) against the
    oracle's DFT to 1e-8 Eh, with stored and with integral-direct J."""
    mol = h2o()
    bs = BasisSet(mol, "6-31g**")
    at = atoms_of(mol)
    obfs = oracle_bfs(bs)
    S, h = O.orc_get1ints(obfs, at)
    e_orc, _, _ = O.dft(at, S, h, O.orc_get2ints(obfs), obfs, 5)
    e_st, _, _ = dft(mol, bfs=bs, ConvCriteria=1e-10, MaxIter=80)
    e_dir, _, _ = dft(mol, bfs=bs, ConvCriteria=1e-10, MaxIter=80, direct=True, schwarz=0.0)
    print("H2O SVWN: GPU stored %.10f direct %.10f oracle %.10f" % (e_st, e_dir, e_orc))
    assert abs(e_st - e_orc) < 1e-8 and abs(e_dir - e_orc) < 1e-8


def test_dft_water_dimer_vs_oracle():
    """(H2O)2 / 6-31G** SVWN, a heteronuclear Becke partition over six
    atoms, against the oracle."""
    mol = geometries.water_cluster(2, seed=4)
    bs = BasisSet(mol, "6-31g**")
    at = atoms_of(mol)
    obfs = oracle_bfs(bs)
    S, h = O.orc_get1ints(obfs, at)
    e_orc, _, _ = O.dft(at, S, h, O.orc_get2ints(obfs), obfs, 10)
    e_gpu, _, _ = dft(mol, bfs=bs, ConvCriteria=1e-10, MaxIter=80, direct=True)
    assert abs(e_gpu - e_orc) < 1e-8
