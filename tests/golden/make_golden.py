"""Regenerate the golden fixtures in this directory.

    make -C oracle ref && python tests/golden/make_golden.py

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


if __name__ == "__main__":
    main()
