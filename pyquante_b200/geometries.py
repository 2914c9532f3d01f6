"""Seeded synthetic molecules for the engine's benchmark and test workloads.

All coordinates are returned in bohr (Molecule units 'bohr');
bohr2ang = 0.529177249 (PyQuante/Constants.py:20).

  water()                   O (0,0,0), H (+-1.4305, 0, 1.1093) bohr
  water_cluster(n, seed)    n waters with water()'s internal geometry,
                            uniformly random orientations (quaternions from
                            seeded normals), O positions uniform in a 9 A
                            cube, any O-O distance < 2.7 A rejected
  alkane(16)                all-trans C16H34: C-C 1.54 A, C-C-C 111 deg,
                            C-H 1.09 A, tetrahedral H
  perturbed(mol, 0.05, s)   every coordinate moved uniformly in +-0.05 bohr
  cluster_batch(count, s)   `count` clusters, k ~ U{1..12} waters each,
                            basis drawn 50/50 from STO-3G / 6-31G*
"""
import numpy as np

from .Constants import ang2bohr
from .Molecule import Molecule

WATER_BOHR = [(8, (0.0, 0.0, 0.0)), (1, (1.4305, 0.0, 1.1093)), (1, (-1.4305, 0.0, 1.1093))]


def water():
    return Molecule("h2o", WATER_BOHR, units="bohr")


def _rotation(q):
    a, b, c, d = q / np.linalg.norm(q)
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def water_cluster(n, seed=0, box_ang=9.0, min_oo_ang=2.7, max_tries=100000):
    rng = np.random.default_rng(seed)
    local = np.array([xyz for _, xyz in WATER_BOHR])
    box = box_ang * ang2bohr
    dmin = min_oo_ang * ang2bohr
    centres = []
    tries = 0
    while len(centres) < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("could not place %d waters in a %.1f A cube" % (n, box_ang))
        c = rng.uniform(0.0, box, size=3)
        if all(np.linalg.norm(c - o) >= dmin for o in centres):
            centres.append(c)
    atoms = []
    for c in centres:
        R = _rotation(rng.standard_normal(4))
        for (z, _), r in zip(WATER_BOHR, local):
            atoms.append((z, tuple(c + R @ r)))
    return Molecule("h2o_%d" % n, atoms, units="bohr")


def alkane(nc=16, cc=1.54, ccc=111.0, ch=1.09):
    """All-trans CnH(2n+2) in the xy plane (angstrom inputs, bohr output)."""
    half = np.radians(ccc) / 2
    dx, dy = cc * np.sin(half), cc * np.cos(half)
    C = np.array([[i * dx, (dy / 2) * (1 if i % 2 else -1), 0.0] for i in range(nc)])
    H = []
    tet = np.radians(109.4712206)
    for i in range(nc):
        nb = [C[j] - C[i] for j in (i - 1, i + 1) if 0 <= j < nc]
        u = [v / np.linalg.norm(v) for v in nb]
        if len(u) == 2:
            b = -(u[0] + u[1])
            b /= np.linalg.norm(b)
            nrm = np.cross(u[0], u[1])
            nrm /= np.linalg.norm(nrm)
            for s in (1, -1):
                H.append(C[i] + ch * (b * np.cos(tet / 2) + s * nrm * np.sin(tet / 2)))
        else:   # methyl: one H anti (in plane), two at +-120 deg about the C-C axis
            ax = u[0]
            perp = np.array([0.0, 1.0 if C[i][1] > 0 else -1.0, 0.0])
            perp -= ax * (perp @ ax)
            perp /= np.linalg.norm(perp)
            w = np.cross(ax, perp)
            for phi in (0.0, 2 * np.pi / 3, -2 * np.pi / 3):
                d = np.cos(np.pi - tet) * (-ax) + np.sin(np.pi - tet) * (np.cos(phi) * perp + np.sin(phi) * w)
                H.append(C[i] + ch * d)
    atoms = [(6, tuple(c * ang2bohr)) for c in C] + [(1, tuple(h * ang2bohr)) for h in H]
    return Molecule("C%dH%d" % (nc, 2 * nc + 2), atoms, units="bohr")


def perturbed(mol, amp=0.05, seed=0):
    rng = np.random.default_rng(seed)
    atoms = [(a.atno, tuple(a.r + rng.uniform(-amp, amp, size=3))) for a in mol.atoms]
    return Molecule(mol.name + "_pert", atoms, units="bohr")


def cluster_batch(count=512, seed=0, kmax=12):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        k = int(rng.integers(1, kmax + 1))
        basis = "sto-3g" if rng.random() < 0.5 else "6-31g*"
        out.append((water_cluster(k, seed=int(rng.integers(0, 2 ** 31))), basis))
    return out
