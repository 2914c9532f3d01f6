"""The synthetic workloads: the seeded generators reproduce the committed
coordinates (tests/golden/geometries.json, written by make_geometries.py)
and obey the construction rules they state (CPU only)."""
import json
import os

import numpy as np

from conftest import GOLDEN
from pyquante_b200 import geometries
from pyquante_b200.Constants import ang2bohr

FIX = json.load(open(os.path.join(GOLDEN, "geometries.json")))


def _xyz(mol):
    return np.array([a.r for a in mol.atoms], dtype=np.float64)


def _same(mol, rows):
    assert [a.atno for a in mol.atoms] == [r[0] for r in rows]
    assert np.abs(_xyz(mol) - np.array([r[1:] for r in rows])).max() < 1e-12


def test_generators_reproduce_the_committed_coordinates():
    _same(geometries.water(), FIX["water"])
    _same(geometries.water_cluster(8, seed=0), FIX["h2o8_seed0"])
    _same(geometries.alkane(16), FIX["c16h34"])
    _same(geometries.perturbed(geometries.water_cluster(4, seed=0), 0.05, seed=7), FIX["h2o4_seed0_pert7"])
    systems = geometries.cluster_batch(512, seed=0)
    for (mol, basis), (k, b, s1, s2) in zip(systems, FIX["batch512_seed0"]):
        r = _xyz(mol)
        assert len(mol.atoms) == 3 * k and basis == b
        assert abs(r.sum() - s1) < 1e-9 and abs((r * r).sum() - s2) < 1e-9 * max(1.0, s2)


def test_water_cluster_rules():
    """Water's internal geometry, O inside the 9 A cube, no O-O under 2.7 A."""
    ref = _xyz(geometries.water())
    d_ref = sorted(np.linalg.norm(ref[i] - ref[j]) for i in range(3) for j in range(i))
    for n, seed in [(8, 0), (12, 3), (4, 0)]:
        r = _xyz(geometries.water_cluster(n, seed=seed)).reshape(n, 3, 3)
        O = r[:, 0]
        assert O.min() >= 0.0 and O.max() <= 9.0 * ang2bohr
        for i in range(n):
            d = sorted(np.linalg.norm(r[i, a] - r[i, b]) for a in range(3) for b in range(a))
            assert np.allclose(d, d_ref, atol=1e-12)
            for j in range(i):
                assert np.linalg.norm(O[i] - O[j]) >= 2.7 * ang2bohr


def test_alkane_rules():
    """All-trans C16H34: C-C 1.54 A, C-C-C 111 deg, C-H 1.09 A, H-C-H
    tetrahedral at the CH2 groups."""
    mol = geometries.alkane(16)
    z = [a.atno for a in mol.atoms]
    assert z.count(6) == 16 and z.count(1) == 34
    r = _xyz(mol) / ang2bohr
    C, H = r[:16], r[16:]
    for i in range(15):
        assert abs(np.linalg.norm(C[i + 1] - C[i]) - 1.54) < 1e-12
    for i in range(1, 15):
        u, v = C[i - 1] - C[i], C[i + 1] - C[i]
        ang = np.degrees(np.arccos(u @ v / np.linalg.norm(u) / np.linalg.norm(v)))
        assert abs(ang - 111.0) < 1e-9
    # every H sits 1.09 A from exactly one carbon; CH3 ends, CH2 in between
    owner = [int(np.argmin(np.linalg.norm(C - h, axis=1))) for h in H]
    for h, c in zip(H, owner):
        assert abs(np.linalg.norm(h - C[c]) - 1.09) < 1e-12
    counts = np.bincount(owner, minlength=16)
    assert counts[0] == counts[15] == 3 and all(counts[1:15] == 2)
    for c in range(1, 15):
        hs = [H[k] - C[c] for k in range(34) if owner[k] == c]
        ang = np.degrees(np.arccos(hs[0] @ hs[1] / np.linalg.norm(hs[0]) / np.linalg.norm(hs[1])))
        assert abs(ang - 109.4712206) < 1e-6


def test_perturbation_and_batch_rules():
    base = geometries.water_cluster(4, seed=0)
    d = _xyz(geometries.perturbed(base, 0.05, seed=7)) - _xyz(base)
    assert np.abs(d).max() <= 0.05 and np.abs(d).max() > 0.03
    systems = geometries.cluster_batch(512, seed=0)
    ks = [len(m.atoms) // 3 for m, _ in systems]
    assert min(ks) == 1 and max(ks) == 12
    nsto = sum(b == "sto-3g" for _, b in systems)
    assert {b for _, b in systems} == {"sto-3g", "6-31g*"} and 200 < nsto < 312
