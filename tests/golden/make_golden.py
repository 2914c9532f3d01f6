"""Regenerate the golden fixtures in this directory.

    make -C oracle ref && python tests/golden/make_golden.py

    python tests/golden/make_golden.py --only-c16h34   # just the C16H34 sample

Sources (nothing here is copied from the reference's files):
  * known answers quoted by the reference's own tests:
      Boys F_0(0)=1, F_0(1), F_{1/2}(6.8)   Src/lib/utils/tests/TestMath.c:18-20
      RHF H2O/6-31G** -76.011751 (+-1e-4)   Tests/h2o.py:16
      RHF H2/6-31G**  -1.082098 (+-1e-6)    Tests/h2.py:16
  * outputs of the reference's own compiled C engine (oracle/_ref, built from
    Src/lib/utils/crys.c) for the integrals of the workloads;
  * 40-digit mpmath values of the Boys function and Rys roots/weights.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import pyq_oracle as O  # noqa: E402

from pyquante_b200 import geometries  # noqa: E402
from pyquante_b200.Basis.p631ss import basis_data as P631SS  # noqa: E402
from pyquante_b200.Basis.sto3g import basis_data as STO3G  # noqa: E402
from pyquante_b200.csrc import gen_tables as G  # noqa: E402

A2B = 1 / 0.529177249


def atoms_of(mol):
    return [(a.atno, tuple(float(c) for c in a.r)) for a in mol.atoms]


def main():
    assert O.ref_available(), "build the reference first: make -C oracle ref"
    crys = O.ref_lib("crys")
    # --- Boys
    boys = {"testmath": [[0, 0.0, 1.0], [0, 1.0, 0.7468241328124271], [0.5, 6.8, 0.073447516533246701]],
            "mpmath": []}
    for m in (0, 1, 2, 4, 8, 12, 16):
        for T in (0.0, 1e-9, 0.3, 1.0, 5.0, 12.7, 25.0, 39.9, 40.1, 60.0, 150.0):
            boys["mpmath"].append([m, T, float(G.boys(m, T))])
    boys["reference_Fgamma"] = [[m, T, crys.Fgamma(float(m), T)] for m, T, _ in boys["mpmath"] if T > 0]
    with open(os.path.join(HERE, "boys.json"), "w") as f:
        json.dump(boys, f, indent=1)
    # --- Rys roots/weights
    rng = np.random.default_rng(11)
    Ts = np.concatenate([[0.0, 1e-8, 0.5, 1.0, 3.0, 10.0, 33.0, 39.99, 47.99, 63.99, 64.0, 100.0, 1e4],
                         rng.uniform(0, 70, 40)])
    rys = {}
    for n in range(1, 6):
        rr, ww = [], []
        for T in Ts:
            r, w = G.rys_exact(n, T)
            rr.append([float(x) for x in r])
            ww.append([float(x) for x in w])
        rys["u%d" % n] = np.array(rr)
        rys["w%d" % n] = np.array(ww)
    np.savez(os.path.join(HERE, "rys.npz"), T=Ts, **rys)
    # --- integrals from the reference's compiled crys
    water = atoms_of(geometries.water())
    bfs = O.build_basis(water, STO3G)
    ints = O.ref_get2ints(bfs)
    S, h = O.orc_get1ints(bfs, water)
    e_c0, _, _ = O.rhf(water, S, h, ints, 5, conv=1e-12)
    Sr, hr = O.ref_get1ints(bfs, water)
    e_c0_refh, _, _ = O.rhf(water, Sr, hr, ints, 5, conv=1e-12)
    np.save(os.path.join(HERE, "eri_sto3g_water.npy"), ints)
    bfs = O.build_basis(water, P631SS)
    ints = O.ref_get2ints(bfs, nproc=8)
    sel = np.sort(rng.choice(len(ints), 6000, replace=False))
    np.savez(os.path.join(HERE, "eri_631ss_water_sample.npz"), index=sel, value=ints[sel])
    S, h = O.orc_get1ints(bfs, water)
    e_w631, _, _ = O.rhf(water, S, h, ints, 5, conv=1e-12)
    # (H2O)8 / 6-31G**: a sample of quartets straight from the reference engine
    cl = atoms_of(geometries.water_cluster(8, seed=0))
    bfs = O.build_basis(cl, P631SS)
    n = len(bfs)
    quart = rng.integers(0, n, size=(4000, 4))
    vals = []
    for i, j, k, l in quart:
        vals.append(O.ref_contr(bfs[i], bfs[j], bfs[k], bfs[l]))
    np.savez(os.path.join(HERE, "eri_631ss_h2o8_sample.npz"), quartets=quart.astype(np.int32), value=np.array(vals))
    # reference test energies (oracle with reference ERIs and exact 1e integrals)
    h2o_t = [(8, (0.0, 0.0, 0.0)), (1, (A2B, 0.0, 0.0)), (1, (0.0, A2B, 0.0))]
    bfs = O.build_basis(h2o_t, P631SS)
    ints = O.ref_get2ints(bfs, nproc=8)
    S, h = O.orc_get1ints(bfs, h2o_t)
    e_h2o, _, _ = O.rhf(h2o_t, S, h, ints, 5, conv=1e-12)
    h2 = [(1, (0.0, 0.0, 0.0)), (1, (1.0, 0.0, 0.0))]
    bfs = O.build_basis(h2, P631SS)
    ints = O.ref_get2ints(bfs)
    S, h = O.orc_get1ints(bfs, h2)
    e_h2, _, _ = O.rhf(h2, S, h, ints, 1, conv=1e-12)
    energies = {
        "water_sto3g": e_c0,
        "water_sto3g_reference_cints_h": e_c0_refh,
        "water_631ss": e_w631,
        "h2o_test_geometry_631ss": e_h2o,
        "h2o_test_literal": -76.011751, "h2o_test_tol": 1e-4,
        "h2_631ss": e_h2,
        "h2_test_literal": -1.082098, "h2_test_tol": 1e-6,
    }
    with open(os.path.join(HERE, "energies.json"), "w") as f:
        json.dump(energies, f, indent=1)
    print(json.dumps(energies, indent=1))


def c16h34_sample(count=3000):
    """C16H34 / 6-31G* (N = 308, Q = 1,132,237,791): quartets straight from
    the reference's compiled crys, drawn (i) where the packed index's
    intermediate ij*(ij+1) no longer fits a 32-bit int (ij >= 46341, the
    range where Src/cints.c:413-425 overflows) and (ii) uniformly over all
    unique quartets.  Its own seeded generator, so regenerating it leaves
    the other fixtures unchanged."""
    from pyquante_b200.Basis.p631s import basis_data as P631S
    bfs = O.build_basis(atoms_of(geometries.alkane(16)), P631S)
    n = len(bfs)
    assert n == 308
    P = n * (n + 1) // 2
    rng = np.random.default_rng(308)

    def split(ij):
        i = int((np.sqrt(8 * ij + 1) - 1) // 2)
        while i * (i + 1) // 2 > ij:
            i -= 1
        while (i + 1) * (i + 2) // 2 <= ij:
            i += 1
        return i, ij - i * (i + 1) // 2

    # functions 304..307 (the only i with ij >= 46341) sit on the last two H
    # atoms; the last carbon (225..239) and the last H atoms are their
    # neighbours, which gives integrals well above zero
    near = np.r_[225:240, 290:308]
    quart = []
    for t in range(count):
        if t < count // 3:
            i = int(rng.integers(304, 308))
            j, k, l = (int(x) for x in rng.choice(near, 3))
            if k < l:
                k, l = l, k
            j = min(j, i)
            if k * (k + 1) // 2 + l > i * (i + 1) // 2 + j:
                k, l = i, j
        else:
            lo = 46341 if t < count * 2 // 3 else 0
            ij = int(rng.integers(lo, P))
            kl = int(rng.integers(0, ij + 1))
            i, j = split(ij)
            k, l = split(kl)
        quart.append((i, j, k, l))
    quart = np.array(quart, dtype=np.int64)
    vals = np.array([O.ref_contr(bfs[i], bfs[j], bfs[k], bfs[l]) for i, j, k, l in quart])
    idx = np.array([O.ijkl2intindex(*q) for q in quart], dtype=np.int64)
    np.savez(os.path.join(HERE, "eri_631s_c16h34_sample.npz"), quartets=quart.astype(np.int32), index=idx,
             value=vals)


if __name__ == "__main__":
    if "--only-c16h34" not in sys.argv:
        main()
    c16h34_sample()
