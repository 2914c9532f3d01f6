"""Host-side check of the generated Obara--Saika / Head-Gordon--Pople class
routines (pyquante_b200/csrc/os_classes.inc, written by csrc/gen_os.py).

The emitted vrr/hrr bodies -- the very expressions the device compiles --
are evaluated in Python for single-primitive shells at random centres and
exponents, and every cartesian component is compared with the oracle's
primitive integral (the HGP restatement in oracle/eri_oracle.c, pinned to
the reference's compiled crys).  The checked-in include must also be what
the generator writes now."""
import os
import random

import numpy as np
import pytest

import pyq_oracle as O
from pyquante_b200.csrc import gen_os
from pyquante_b200.csrc.gen_tables import boys

HERE = os.path.dirname(os.path.abspath(__file__))
INC = os.path.join(os.path.dirname(HERE), "pyquante_b200", "csrc", "os_classes.inc")


def _prim(origin, powers, alpha):
    return O.BF(origin, powers, [(alpha, 1.0)])


def _generated_quartet(cls, A, B, C, D, a, b, c, d):
    """(ab|cd) of unnormalised primitives through the emitted code."""
    LA, LB, LC, LD = cls
    lines, _, _ = gen_os.emit_class(*cls)
    vrr, hrr = gen_os.as_python(lines)
    A, B, C, D = (np.array(x, dtype=float) for x in (A, B, C, D))
    z, e = a + b, c + d
    P = (a * A + b * B) / z
    Q = (c * C + d * D) / e
    PQ = P - Q
    T = z * e / (z + e) * PQ @ PQ
    pre = 2 * np.pi ** 2.5 / (z * e * np.sqrt(z + e)) * np.exp(-a * b / z * (A - B) @ (A - B)) * \
        np.exp(-c * d / e * (C - D) @ (C - D))
    F = [pre * float(boys(m, T)) for m in range(sum(cls) + 1)]
    rz, re = e / (z + e), z / (z + e)
    g = {"PA": P - A, "QC": Q - C, "WP": -rz * PQ, "WQ": re * PQ, "oo2z": 0.5 / z, "oo2e": 0.5 / e,
         "rz": rz, "re": re, "oo2ze": 0.5 / (z + e)}
    v = [0.0] * len(gen_os.targets(*cls))
    vrr(g, F, v)
    out = [0.0] * (len(gen_os.carts(LA)) * len(gen_os.carts(LB)) * len(gen_os.carts(LC)) * len(gen_os.carts(LD)))
    hrr(A - B, C - D, v, out)
    return out


@pytest.mark.parametrize("cls", gen_os.OS_CLASSES + [(2, 1, 1, 1), (2, 2, 2, 2)])
def test_generated_recurrences_match_the_oracle(cls):
    """Every class the kernels use, plus two larger ones that exercise every
    recurrence term of the generator."""
    rnd = random.Random(sum(cls) * 7 + cls[0])
    LA, LB, LC, LD = cls
    for trial in range(3 if sum(cls) <= 5 else 1):
        A, B, C, D = ([rnd.uniform(-1.5, 1.5) for _ in range(3)] for _ in range(4))
        a, b, c, d = (rnd.uniform(0.15, 4.0) for _ in range(4))
        got = _generated_quartet(cls, A, B, C, D, a, b, c, d)
        k = 0
        for pa in gen_os.carts(LA):
            for pb in gen_os.carts(LB):
                for pc in gen_os.carts(LC):
                    for pd in gen_os.carts(LD):
                        fs = [_prim(A, pa, a), _prim(B, pb, b), _prim(C, pc, c), _prim(D, pd, d)]
                        norm = np.prod([f.pnorms[0] for f in fs])
                        ref = O.orc_contr(*fs) / norm
                        assert abs(got[k] - ref) <= 1e-12 * max(1.0, abs(ref)), (cls, trial, pa, pb, pc, pd)
                        k += 1


def test_checked_in_include_is_current():
    text, _ = gen_os.source()
    with open(INC) as f:
        assert f.read() == text
