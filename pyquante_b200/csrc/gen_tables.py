"""Generate the device lookup tables used by the ERI kernels.

Writes ``rys_tables.inc`` next to this file.  Run once (takes ~1 min):

    python -m pyquante_b200.csrc.gen_tables              # rys_tables.inc
    python -m pyquante_b200.csrc.gen_tables --boys-top   # boys_top.inc

Two tables are produced, both from 40-digit mpmath arithmetic:

Boys function
    F_m(T) = int_0^1 t^(2m) exp(-T t^2) dt on the grid T_k = k/16,
    k = 0..BOYS_NGRID-1, orders m = 0..BOYS_NORD-1.  The kernels evaluate
    F_mmax(T) by an 8-term Taylor expansion about the nearest grid point
    (dF_m/dT = -F_(m+1)) and then recur downward,
    F_m = (2T F_(m+1) + exp(-T)) / (2m+1).  For T >= BOYS_TMAX they use
    F_0 = sqrt(pi/T)/2 and the upward recursion.

Rys roots and weights
    For n = 1..RYS_NMAX roots, the n-point Gauss rule for the weight
    exp(-T u)/(2 sqrt(u)) on u = t^2 in [0,1] (so sum w_i = F_0(T) and
    sum w_i u_i^k = F_k(T) for k < 2n).  Nodes and weights come from the
    Golub--Welsch eigenproblem of the Jacobi matrix built from the moments
    F_0..F_2n(T) (Hankel Cholesky), in 40-digit arithmetic so the
    ill-conditioning of the moment map is irrelevant.  Each root u_i(T) and
    weight w_i(T) is fitted on unit intervals [j, j+1) of T by a degree-13
    Chebyshev series (14 coefficients, evaluated by Clenshaw on device)
    for T < RYS_TASYM[n]; above that the large-T limit is used:
    u_i = s_i/T, w_i = W_i/sqrt(T) with (s_i, 2 W_i) the generalised
    Gauss--Laguerre (alpha = -1/2) nodes and weights.  RYS_TASYM[n] is where
    that limit is exact to < 2e-15 relative.  The table stores, per (n,
    interval, root), the 14 coefficient pairs (root_k, weight_k) interleaved.

This replaces the GAMESS piecewise fits in the reference's Src/crys.c:99-1438
(Roots/Root123/Root4/Root5) with tables of this project's own construction.
"""
import os

import mpmath as mp

mp.mp.dps = 40

BOYS_NORD = 24          # orders stored: m = 0..23 (mmax 16 + 8 Taylor terms)
BOYS_STEP_INV = 16      # grid spacing 1/16
BOYS_TMAX = 40.0
BOYS_NGRID = int(BOYS_TMAX * BOYS_STEP_INV) + 2

RYS_NMAX = 5
RYS_DEG = 13
RYS_NCOEF = RYS_DEG + 1
RYS_TASYM = {1: 40, 2: 48, 3: 52, 4: 58, 5: 64}


def boys(m, T):
    T = mp.mpf(T)
    if T == 0:
        return mp.mpf(1) / (2 * m + 1)
    return mp.gammainc(m + mp.mpf(1) / 2, 0, T) / (2 * T ** (m + mp.mpf(1) / 2))


def _gauss_from_moments(mu, n):
    H = mp.matrix(n + 1, n + 1)
    for i in range(n + 1):
        for j in range(n + 1):
            H[i, j] = mu[i + j]
    R = mp.cholesky(H).T
    J = mp.matrix(n, n)
    for j in range(n):
        J[j, j] = R[j, j + 1] / R[j, j] - (R[j - 1, j] / R[j - 1, j - 1] if j > 0 else 0)
        if j < n - 1:
            J[j, j + 1] = J[j + 1, j] = R[j + 1, j + 1] / R[j, j]
    E, Qv = mp.eigsy(J)
    idx = sorted(range(n), key=lambda i: E[i])
    return [E[i] for i in idx], [mu[0] * Qv[0, i] ** 2 for i in idx]


def rys_exact(n, T):
    """(roots u_i, weights w_i) of the n-point Rys rule at T, 40 digits."""
    return _gauss_from_moments([boys(k, T) for k in range(2 * n + 1)], n)


def laguerre_half(n):
    """Nodes s_i and weights W_i with int_0^inf f(s) s^-1/2 e^-s ds / 2 = sum W_i f(s_i)."""
    s, w = _gauss_from_moments([mp.gamma(k + mp.mpf(1) / 2) for k in range(2 * n + 1)], n)
    return s, [wi / 2 for wi in w]


def _cheb_fit(f, a, b, deg):
    N = deg + 1
    xs = [mp.cos(mp.pi * (j + mp.mpf(1) / 2) / N) for j in range(N)]
    vals = [f(a + (b - a) * (x + 1) / 2) for x in xs]
    out = []
    for k in range(N):
        s = mp.fsum(vals[j][0] * mp.cos(mp.pi * k * (j + mp.mpf(1) / 2) / N) for j in range(N))
        out.append(s)
    return xs, vals


def build_rys():
    """coef[n][interval][2n][NCOEF] (roots and weights interleaved r0,w0,r1,w1..)."""
    tables = {}
    for n in range(1, RYS_NMAX + 1):
        N = RYS_NCOEF
        xs = [mp.cos(mp.pi * (j + mp.mpf(1) / 2) / N) for j in range(N)]
        per_n = []
        for iv in range(RYS_TASYM[n]):
            sols = [rys_exact(n, iv + (x + 1) / 2) for x in xs]
            funcs = []
            for r in range(n):
                for kind in (0, 1):
                    vals = [sol[kind][r] for sol in sols]
                    cs = []
                    for k in range(N):
                        s = mp.fsum(vals[j] * mp.cos(mp.pi * k * (j + mp.mpf(1) / 2) / N) for j in range(N))
                        cs.append(2 * s / N)
                    cs[0] /= 2
                    funcs.append([float(c) for c in cs])
            per_n.append(funcs)
        tables[n] = per_n
    return tables


def clenshaw(c, x):
    b1 = b2 = 0.0
    for ck in reversed(c[1:]):
        b1, b2 = 2.0 * x * b1 - b2 + ck, b1
    return x * b1 - b2 + c[0]


def check_rys(tables, asym, samples=40):
    import random
    rnd = random.Random(7)
    worst = {}
    for n in range(1, RYS_NMAX + 1):
        e = 0.0
        Ts = [rnd.uniform(0, RYS_TASYM[n] + 10) for _ in range(samples)] + [0.0, 1e-9, RYS_TASYM[n] - 1e-9]
        for T in Ts:
            r, w = rys_exact(n, T)
            if T < RYS_TASYM[n]:
                iv = int(T)
                x = 2.0 * (T - iv) - 1.0
                fn = tables[n][iv]
                got = [(clenshaw(fn[2 * i], x), clenshaw(fn[2 * i + 1], x)) for i in range(n)]
            else:
                s, W = asym[n]
                got = [(float(s[i]) / T, float(W[i]) / T ** 0.5) for i in range(n)]
            for i in range(n):
                e = max(e, abs(got[i][0] - float(r[i])) / float(r[i]), abs(got[i][1] - float(w[i])) / float(w[i]))
        worst[n] = e
    return worst


def main():
    here = os.path.dirname(os.path.abspath(__file__))
    boys_tab = [[float(boys(m, mp.mpf(k) / BOYS_STEP_INV)) for m in range(BOYS_NORD)] for k in range(BOYS_NGRID)]
    rys = build_rys()
    asym = {n: laguerre_half(n) for n in range(1, RYS_NMAX + 1)}
    worst = check_rys(rys, asym)
    lines = ["// Generated by gen_tables.py -- do not edit.",
             "// Max relative error of the fitted Rys roots/weights against 40-digit",
             "// Golub--Welsch (random T): " + ", ".join("n=%d %.1e" % (n, worst[n]) for n in sorted(worst)),
             "// Includers define PQB_TABQ / PQB_CTABQ (storage qualifiers of the big",
             "// and the small arrays), e.g. __device__ const / __constant__ const.",
             "#pragma once",
             "#define PQB_BOYS_NORD %d" % BOYS_NORD,
             "#define PQB_BOYS_STEP_INV %d" % BOYS_STEP_INV,
             "#define PQB_BOYS_TMAX %.1f" % BOYS_TMAX,
             "#define PQB_BOYS_NGRID %d" % BOYS_NGRID,
             "#define PQB_RYS_NMAX %d" % RYS_NMAX,
             "#define PQB_RYS_NCOEF %d" % RYS_NCOEF]
    off = 0
    offs = []
    for n in range(1, RYS_NMAX + 1):
        offs.append(off)
        off += RYS_TASYM[n] * 2 * n * RYS_NCOEF
    lines.append("#define PQB_RYS_TABLE_SIZE %d" % off)
    lines.append("PQB_CTABQ int pqb_rys_tasym[%d] = {0, %s};" %
                 (RYS_NMAX + 1, ", ".join(str(RYS_TASYM[n]) for n in range(1, RYS_NMAX + 1))))
    lines.append("PQB_CTABQ int pqb_rys_offset[%d] = {0, %s};" % (RYS_NMAX + 1, ", ".join(map(str, offs))))
    lines.append("PQB_CTABQ double pqb_rys_asym_root[%d][%d] = {" % (RYS_NMAX + 1, RYS_NMAX))
    lines.append("  {0},")
    for n in range(1, RYS_NMAX + 1):
        lines.append("  {" + ", ".join("%.17e" % float(s) for s in asym[n][0]) + "},")
    lines.append("};")
    lines.append("PQB_CTABQ double pqb_rys_asym_weight[%d][%d] = {" % (RYS_NMAX + 1, RYS_NMAX))
    lines.append("  {0},")
    for n in range(1, RYS_NMAX + 1):
        lines.append("  {" + ", ".join("%.17e" % float(w) for w in asym[n][1]) + "},")
    lines.append("};")
    # per (n, interval, root): the 14 (root, weight) coefficient pairs
    # interleaved, 224 bytes, so a lane reads both series with 256-bit loads
    lines.append("PQB_TABQ __align__(64) double pqb_rys_coef[PQB_RYS_TABLE_SIZE] = {")
    for n in range(1, RYS_NMAX + 1):
        for iv, funcs in enumerate(rys[n]):
            for r in range(n):
                cu, cw = funcs[2 * r], funcs[2 * r + 1]
                lines.append("  " + ", ".join("%.17e, %.17e" % (a, b) for a, b in zip(cu, cw)) + ",")
    lines.append("};")
    # FP32 copy for the mixed-precision kernels: per (n, interval, root) the
    # first 7 coefficient pairs (the rest sum to < 1.1e-8 relative) and a zero
    # pair, 64 bytes: two 256-bit loads
    lines.append("#define PQB_RYS_NCOEF_F32 7")
    lines.append("PQB_TABQ __align__(64) float pqb_rys_coef_f32[PQB_RYS_TABLE_SIZE / 14 * 16 / 2] = {")
    for n in range(1, RYS_NMAX + 1):
        for iv, funcs in enumerate(rys[n]):
            for r in range(n):
                cu, cw = funcs[2 * r], funcs[2 * r + 1]
                pairs = [(cu[k], cw[k]) for k in range(7)] + [(0.0, 0.0)]
                lines.append("  " + ", ".join("%.9ef, %.9ef" % (a, b) for a, b in pairs) + ",")
    lines.append("};")
    lines.append("PQB_TABQ double pqb_boys_tab[PQB_BOYS_NGRID * PQB_BOYS_NORD] = {")
    for row in boys_tab:
        lines.append("  " + ", ".join("%.17e" % v for v in row) + ",")
    lines.append("};")
    with open(os.path.join(here, "rys_tables.inc"), "w") as f:
        f.write("\n".join(lines) + "\n")
    print("worst relative error:", worst)


# Grid of the compact Boys rows of the Fock-build kernels: T_k = k/32,
# k = 0..BOYSROW_NGRID-1, up to BOYS_TMAX (large-T forms beyond).
BOYSROW_STEP_INV = 32
BOYSROW_NGRID = int(BOYS_TMAX * BOYSROW_STEP_INV) + 2


# 16-byte Boys rows: {F_top(T_k), exp(-T_k)} at T_k = k/32 for top = 7 and
# 10 (and an 8-byte single-precision copy for top = 7).  The device rebuilds F_j(T_k), j < top, by the downward recursion
# F_j = (2 T_k F_(j+1) + exp(-T_k)) / (2j+1) (stable: each step keeps or
# shrinks the relative error) and then sums the same Taylor series in
# d = T_k - T as with the 64-byte rows, from a table a quarter of the size.
BOYSTOP_ORDERS = (7, 10)


def main_boys_top():
    here = os.path.dirname(os.path.abspath(__file__))
    lines = ["// Generated by gen_tables.py --boys-top -- do not edit.",
             "// Row k at T_k = k/%d (40-digit mpmath): {F_top(T_k), exp(-T_k)}, top = 7 and 10; FP32 copy for top = 7."
             % BOYSROW_STEP_INV,
             "#pragma once",
             "#define PQB_BOYSROW_STEP_INV %d" % BOYSROW_STEP_INV,
             "#define PQB_BOYSROW_NGRID %d" % BOYSROW_NGRID,
             "#define PQB_BOYSROW_TMAX %.1f" % BOYS_TMAX]
    for top in BOYSTOP_ORDERS:
        lines.append("PQB_TABQ __align__(16) double pqb_boys_top%d[PQB_BOYSROW_NGRID * 2] = {" % top)
        for k in range(BOYSROW_NGRID):
            T = mp.mpf(k) / BOYSROW_STEP_INV
            lines.append("  %.17e, %.17e," % (float(boys(top, T)), float(mp.exp(-T))))
        lines.append("};")
    # single precision, top = 7, for the FP32 lists of the mixed mode
    lines.append("PQB_TABQ __align__(8) float pqb_boys_top7_f32[PQB_BOYSROW_NGRID * 2] = {")
    for k in range(BOYSROW_NGRID):
        T = mp.mpf(k) / BOYSROW_STEP_INV
        lines.append("  %.9ef, %.9ef," % (float(boys(7, T)), float(mp.exp(-T))))
    lines.append("};")
    with open(os.path.join(here, "boys_top.inc"), "w") as f:
        f.write("\n".join(lines) + "\n")


if __name__ == "__main__":
    import sys
    if "--boys-top" in sys.argv:
        main_boys_top()
    else:
        main()
