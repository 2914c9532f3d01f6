"""The 194-point Lebedev--Laikov angular quadrature (V. I. Lebedev and
D. N. Laikov, Doklady Mathematics 59, 477 (1999)): the angular rule of the
default DFT grid of the reference (PyQuante/AtomicGrid.py:85-99 takes
Lebedev[194] for every radial shell; the points are listed in
PyQuante/Lebedev.py:754-950).

The rule is octahedrally invariant: its 194 points are the orbits
    a1  (1, 0, 0)                 6 points
    a2  (0, 1, 1)/sqrt(2)        12
    a3  (1, 1, 1)/sqrt(3)         8
    b   (l, l, m), m = sqrt(1 - 2 l^2)     4 orbits of 24
    c   (p, q, 0), q = sqrt(1 - p^2)       1 orbit of 24
    d   (r, s, t), t = sqrt(1 - r^2 - s^2) 1 orbit of 48
with one weight per orbit, and it integrates every polynomial of degree
<= 23 on the sphere exactly.  PARAMS holds the published orbit parameters
and weights, refined here to full double precision: ``refine()`` solves the
exactness conditions for the even monomials x^2i y^2j z^2k (i + j + k <= 11,
sphere averages (2i-1)!!(2j-1)!!(2k-1)!!/(2n+1)!!) by Gauss--Newton in
40-digit arithmetic, starting from the published 12-digit values.

    python -m pyquante_b200.Lebedev     # re-run the refinement, print PARAMS
"""
import itertools

import numpy as np

# published 12-digit values (weights sum to 1; the reference tabulates the same)
PUBLISHED = dict(
    w_a1=0.001782340447, w_a2=0.005716905950, w_a3=0.005573383179,
    b=[(0.129933544765, 0.004106777028), (0.289246562758, 0.005158237712),
       (0.444693317872, 0.005518771467), (0.671297344270, 0.005608704083)],
    c=(0.938319218138, 0.005051846065),
    d=(0.836036015482, 0.525118572444, 0.005530248916),
)

# the same, refined by refine() (max residual of the exactness conditions
# 1.4e-42 in 40-digit arithmetic), rounded to double precision
PARAMS = {'w_a1': 0.0017823404472446112, 'w_a2': 0.005716905949977102, 'w_a3': 0.005573383178848738,
          'b': [(0.12993354476500668, 0.004106777028169394), (0.28924656275754385, 0.005158237711805383),
                (0.4446933178717437, 0.0055187714672736135), (0.6712973442695226, 0.005608704082587997)],
          'c': (0.9383192181375916, 0.005051846064614809),
          'd': (0.8360360154824589, 0.525118572443642, 0.0055302489162330935)}


def _perms_signs(v):
    """All points of the orbit of v under permutations and sign changes."""
    pts = set()
    for p in itertools.permutations(v):
        for s in itertools.product((1, -1), repeat=3):
            pts.add(tuple(si * pi for si, pi in zip(s, p)))
    return sorted(pts)


def orbits(prm, sqrt):
    """[(points, weight)] of the rule for parameters prm (sqrt: the square
    root to use, so the same code serves floats and mpmath numbers)."""
    one = prm["w_a1"] * 0 + 1
    out = [(_perms_signs((one, 0 * one, 0 * one)), prm["w_a1"]),
           (_perms_signs((0 * one, one / sqrt(2 * one), one / sqrt(2 * one))), prm["w_a2"]),
           (_perms_signs((one / sqrt(3 * one),) * 3), prm["w_a3"])]
    for l, w in prm["b"]:
        out.append((_perms_signs((l, l, sqrt(1 - 2 * l * l))), w))
    p, w = prm["c"]
    out.append((_perms_signs((p, sqrt(1 - p * p), 0 * one)), w))
    r, s, w = prm["d"]
    out.append((_perms_signs((r, s, sqrt(1 - r * r - s * s))), w))
    return out


def points(prm=None):
    """(194, 4) array of x, y, z, w."""
    prm = prm or PARAMS
    rows = [(x, y, z, w) for pts, w in orbits(prm, np.sqrt) for x, y, z in pts]
    assert len(rows) == 194
    return np.array(rows, dtype=np.float64)


def _dfact(n):
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return r


def monomials(nmax=11):
    return [(i, j, k) for n in range(nmax + 1) for i in range(n, -1, -1) for j in range(min(i, n - i), -1, -1)
            for k in [n - i - j] if k <= j]


def exact_average(i, j, k):
    """(1/4pi) * integral of x^2i y^2j z^2k over the unit sphere."""
    return _dfact(2 * i - 1) * _dfact(2 * j - 1) * _dfact(2 * k - 1) / _dfact(2 * (i + j + k) + 1)


def refine(start=None, iters=4, dps=40):
    import mpmath as mp
    mp.mp.dps = dps
    start = start or PUBLISHED

    def pack(prm):
        v = [prm["w_a1"], prm["w_a2"], prm["w_a3"]]
        for l, w in prm["b"]:
            v += [l, w]
        v += list(prm["c"]) + list(prm["d"])
        return [mp.mpf(repr(float(x))) for x in v]

    def unpack(v):
        return dict(w_a1=v[0], w_a2=v[1], w_a3=v[2], b=[(v[3 + 2 * q], v[4 + 2 * q]) for q in range(4)],
                    c=(v[11], v[12]), d=(v[13], v[14], v[15]))

    mons = monomials()
    target = [mp.mpf(_dfact(2 * i - 1) * _dfact(2 * j - 1) * _dfact(2 * k - 1)) / _dfact(2 * (i + j + k) + 1)
              for i, j, k in mons]

    def resid(v):
        orb = orbits(unpack(v), mp.sqrt)
        out = []
        for (i, j, k), t in zip(mons, target):
            s = mp.mpf(0)
            for pts, w in orb:
                s += w * mp.fsum(x ** (2 * i) * y ** (2 * j) * z ** (2 * k) for x, y, z in pts)
            out.append(s - t)
        return mp.matrix(out)

    v = pack(start)
    for _ in range(iters):
        r = resid(v)
        h = mp.mpf(10) ** (-dps // 2)
        Jm = mp.matrix(len(r), len(v))
        for c in range(len(v)):
            vp = list(v)
            vp[c] += h
            rc = resid(vp)
            for rr in range(len(r)):
                Jm[rr, c] = (rc[rr] - r[rr]) / h
        step = mp.lu_solve(Jm.T * Jm, Jm.T * r)
        v = [v[c] - step[c] for c in range(len(v))]
    return unpack([float(x) for x in v]), float(mp.norm(resid(v), p=mp.inf))


if __name__ == "__main__":
    prm, res = refine()
    print("max residual %.3e" % res)
    print(repr(prm))
