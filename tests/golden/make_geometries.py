"""Write the coordinates of the benchmark workloads to geometries.json.

    python tests/golden/make_geometries.py

The workloads are synthetic: pyquante_b200.geometries builds them from
seeded rules.  The file records what those rules give (bohr), so that a
change of generator or of numpy's random streams shows up as a test
failure instead of a silently different benchmark input.
  water            O (0,0,0), H (+-1.4305, 0, 1.1093) bohr
  h2o8_seed0       (H2O)8, 9 A cube, O-O >= 2.7 A  (bench.py default workload)
  c16h34           all-trans C16H34                (bench.py --workload c16h34)
  h2o4_seed0_pert7 (H2O)4 perturbed +-0.05 bohr    (bench.py --workload h2o4-grad)
  batch512_seed0   per cluster: water count, basis, coordinate sum and sum of
                   squares                         (bench.py --workload batch)
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from pyquante_b200 import geometries  # noqa: E402


def atoms(mol):
    return [[int(a.atno)] + [float(c) for c in a.r] for a in mol.atoms]


def batch_summary(systems):
    out = []
    for mol, basis in systems:
        r = np.array([a.r for a in mol.atoms], dtype=np.float64)
        out.append([len(mol.atoms) // 3, basis, float(r.sum()), float((r * r).sum())])
    return out


def build():
    return {
        "units": "bohr",
        "water": atoms(geometries.water()),
        "h2o8_seed0": atoms(geometries.water_cluster(8, seed=0)),
        "c16h34": atoms(geometries.alkane(16)),
        "h2o4_seed0_pert7": atoms(geometries.perturbed(geometries.water_cluster(4, seed=0), 0.05, seed=7)),
        "batch512_seed0": batch_summary(geometries.cluster_batch(512, seed=0)),
    }


if __name__ == "__main__":
    data = build()
    parts = ['"units": "bohr"']
    for key, rows in data.items():
        if key != "units":
            parts.append('"%s": [\n%s\n]' % (key, ",\n".join(json.dumps(r) for r in rows)))
    with open(os.path.join(HERE, "geometries.json"), "w") as f:
        f.write("{\n" + ",\n".join(parts) + "\n}\n")
