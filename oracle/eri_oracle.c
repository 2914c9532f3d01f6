/* CPU oracle — test infrastructure only (see oracle.h for what it restates).
 * Only tests, the smoke check and the bench's CPU-baseline leg may load it. */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ---------------------------------------------------------------- Boys --
 * F_m(T) = int_0^1 t^{2m} exp(-T t^2) dt.
 * Replaces the NR incomplete gamma of Src/chgp.c:619-690 / Src/cints.c:340-411
 * by the convergent series F_m(T) = e^{-T} sum_k (2T)^k / ((2m+1)(2m+3)...(2m+2k+1))
 * in long double (all terms positive, so no cancellation), and for T > 80 by
 * F_0 = sqrt(pi/T) erf(sqrt T)/2 followed by the upward recursion
 * F_{m+1} = ((2m+1) F_m - e^{-T}) / (2T), which is stable for T >> m. */
static long double boys_ld(int m, long double T)
{
    if (T <= 80.0L) {
        long double term = 1.0L / (2 * m + 1), sum = term;
        for (int k = 1; k < 4000; k++) {
            term *= 2.0L * T / (2 * m + 2 * k + 1);
            sum += term;
            if (term < sum * 1e-22L) break;
        }
        return expl(-T) * sum;
    }
    long double f = 0.5L * sqrtl(M_PI / T) * erfl(sqrtl(T)), e = expl(-T);
    for (int k = 0; k < m; k++) f = ((2 * k + 1) * f - e) / (2.0L * T);
    return f;
}

double orc_boys(int m, double T) { return (double)boys_ld(m, (long double)T); }

/* ------------------------------------------------------- packed index --
 * Src/cints.c:413-425 ordering, 64-bit arithmetic. */
int64_t orc_ijkl2intindex(int64_t i, int64_t j, int64_t k, int64_t l)
{
    int64_t t;
    if (i < j) { t = i; i = j; j = t; }
    if (k < l) { t = k; k = l; l = t; }
    int64_t ij = i * (i + 1) / 2 + j, kl = k * (k + 1) / 2 + l;
    if (ij < kl) { t = ij; ij = kl; kl = t; }
    return ij * (ij + 1) / 2 + kl;
}

/* ------------------------------------------------------------ HGP ERI --
 * Obara--Saika VRR (a0|c0)^(m) and HGP HRR, the scheme of Src/chgp.c:78-419,
 * memoised on (cartesian a, cartesian c, m) with a generation stamp so no
 * table has to be cleared between primitive quartets. */
#define ORC_MAXL 8                                    /* per side, a or c */
#define ORC_NCART ((ORC_MAXL + 1) * (ORC_MAXL + 2) * (ORC_MAXL + 3) / 6)
#define ORC_MAXM (2 * ORC_MAXL + 2)

static double memo_v[ORC_NCART][ORC_NCART][ORC_MAXM];
static unsigned memo_g[ORC_NCART][ORC_NCART][ORC_MAXM];
static unsigned memo_gen = 0;

typedef struct {
    double PA[3], QC[3], WP[3], WQ[3];
    double oo2z, oo2e, oo2ze, rz, re; /* 1/2zeta, 1/2eta, 1/2(zeta+eta), eta/(z+e), zeta/(z+e) */
    double F[ORC_MAXM];               /* prefactor * F_m(T) */
} vrr_ctx;

static inline int cart_index(const int *l)
{
    int n = l[0] + l[1] + l[2];
    return n * (n + 1) * (n + 2) / 6 + (n - l[0]) * (n - l[0] + 1) / 2 + (n - l[0] - l[1]);
}

static double vrr(const vrr_ctx *c, const int *a, const int *cc, int m)
{
    int ia = cart_index(a), ic = cart_index(cc);
    if (memo_g[ia][ic][m] == memo_gen) return memo_v[ia][ic][m];
    double v;
    int i;
    if (a[0] + a[1] + a[2] > 0) {
        i = a[0] ? 0 : (a[1] ? 1 : 2);
        int a1[3] = {a[0], a[1], a[2]};
        a1[i]--;
        v = c->PA[i] * vrr(c, a1, cc, m) + c->WP[i] * vrr(c, a1, cc, m + 1);
        if (a1[i] > 0) {
            int a2[3] = {a1[0], a1[1], a1[2]};
            a2[i]--;
            v += a1[i] * c->oo2z * (vrr(c, a2, cc, m) - c->rz * vrr(c, a2, cc, m + 1));
        }
        if (cc[i] > 0) {
            int c1[3] = {cc[0], cc[1], cc[2]};
            c1[i]--;
            v += cc[i] * c->oo2ze * vrr(c, a1, c1, m + 1);
        }
    } else if (cc[0] + cc[1] + cc[2] > 0) {
        i = cc[0] ? 0 : (cc[1] ? 1 : 2);
        int c1[3] = {cc[0], cc[1], cc[2]};
        c1[i]--;
        v = c->QC[i] * vrr(c, a, c1, m) + c->WQ[i] * vrr(c, a, c1, m + 1);
        if (c1[i] > 0) {
            int c2[3] = {c1[0], c1[1], c1[2]};
            c2[i]--;
            v += c1[i] * c->oo2e * (vrr(c, a, c2, m) - c->re * vrr(c, a, c2, m + 1));
        }
    } else {
        v = c->F[m];
    }
    memo_g[ia][ic][m] = memo_gen;
    memo_v[ia][ic][m] = v;
    return v;
}

static double hrr(const vrr_ctx *c, const double *AB, const double *CD, const int *a, const int *b,
                  const int *cc, const int *d)
{
    for (int i = 0; i < 3; i++)
        if (b[i] > 0) {
            int a1[3] = {a[0], a[1], a[2]}, b1[3] = {b[0], b[1], b[2]};
            a1[i]++;
            b1[i]--;
            return hrr(c, AB, CD, a1, b1, cc, d) + AB[i] * hrr(c, AB, CD, a, b1, cc, d);
        }
    for (int i = 0; i < 3; i++)
        if (d[i] > 0) {
            int c1[3] = {cc[0], cc[1], cc[2]}, d1[3] = {d[0], d[1], d[2]};
            c1[i]++;
            d1[i]--;
            return hrr(c, AB, CD, a, b, c1, d1) + CD[i] * hrr(c, AB, CD, a, b, cc, d1);
        }
    return vrr(c, a, cc, 0);
}

double orc_prim_eri(const double *A, double na, const int *la, double aa,
                    const double *B, double nb, const int *lb, double ab,
                    const double *C, double nc, const int *lc, double ac,
                    const double *D, double nd, const int *ld, double ad)
{
    vrr_ctx c;
    double zeta = aa + ab, eta = ac + ad, P[3], Q[3], W[3], AB[3], CD[3], rab2 = 0, rcd2 = 0, rpq2 = 0;
    for (int i = 0; i < 3; i++) {
        P[i] = (aa * A[i] + ab * B[i]) / zeta;
        Q[i] = (ac * C[i] + ad * D[i]) / eta;
        W[i] = (zeta * P[i] + eta * Q[i]) / (zeta + eta);
        AB[i] = A[i] - B[i];
        CD[i] = C[i] - D[i];
        rab2 += AB[i] * AB[i];
        rcd2 += CD[i] * CD[i];
        rpq2 += (P[i] - Q[i]) * (P[i] - Q[i]);
        c.PA[i] = P[i] - A[i];
        c.QC[i] = Q[i] - C[i];
        c.WP[i] = W[i] - P[i];
        c.WQ[i] = W[i] - Q[i];
    }
    c.oo2z = 0.5 / zeta;
    c.oo2e = 0.5 / eta;
    c.oo2ze = 0.5 / (zeta + eta);
    c.rz = eta / (zeta + eta);
    c.re = zeta / (zeta + eta);
    int ltot = la[0] + la[1] + la[2] + lb[0] + lb[1] + lb[2] + lc[0] + lc[1] + lc[2] + ld[0] + ld[1] + ld[2];
    double T = zeta * eta / (zeta + eta) * rpq2;
    /* 2 pi^{5/2} / (zeta eta sqrt(zeta+eta)) exp(-ab/zeta Rab^2 - cd/eta Rcd^2)  (Src/chgp.c:270-276) */
    double pre = 2.0 * pow(M_PI, 2.5) / (zeta * eta * sqrt(zeta + eta)) *
                 exp(-aa * ab / zeta * rab2 - ac * ad / eta * rcd2);
    for (int m = 0; m <= ltot; m++) c.F[m] = pre * orc_boys(m, T);
    if (++memo_gen == 0) {
        memset(memo_g, 0, sizeof(memo_g));
        memo_gen = 1;
    }
    return na * nb * nc * nd * hrr(&c, AB, CD, la, lb, lc, ld);
}

double orc_contr_eri(int lena, const double *aexps, const double *acoefs, const double *anorms,
                     const double *A, const int *la,
                     int lenb, const double *bexps, const double *bcoefs, const double *bnorms,
                     const double *B, const int *lb,
                     int lenc, const double *cexps, const double *ccoefs, const double *cnorms,
                     const double *C, const int *lc,
                     int lend, const double *dexps, const double *dcoefs, const double *dnorms,
                     const double *D, const int *ld)
{
    /* contraction as Src/crys.c:34-54: sum c_a c_b c_c c_d (prim ERI with prim norms) */
    double v = 0;
    for (int p = 0; p < lena; p++)
        for (int q = 0; q < lenb; q++)
            for (int r = 0; r < lenc; r++)
                for (int s = 0; s < lend; s++)
                    v += acoefs[p] * bcoefs[q] * ccoefs[r] * dcoefs[s] *
                         orc_prim_eri(A, anorms[p], la, aexps[p], B, bnorms[q], lb, bexps[q],
                                      C, cnorms[r], lc, cexps[r], D, dnorms[s], ld, dexps[s]);
    return v;
}

static double bf_coulomb(const double *origin, const int64_t *powers, const int64_t *off,
                         const double *exps, const double *coefs, const double *pnorms, const double *norms,
                         int64_t a, int64_t b, int64_t c, int64_t d)
{
    int la[3] = {(int)powers[3 * a], (int)powers[3 * a + 1], (int)powers[3 * a + 2]};
    int lb[3] = {(int)powers[3 * b], (int)powers[3 * b + 1], (int)powers[3 * b + 2]};
    int lc[3] = {(int)powers[3 * c], (int)powers[3 * c + 1], (int)powers[3 * c + 2]};
    int ld[3] = {(int)powers[3 * d], (int)powers[3 * d + 1], (int)powers[3 * d + 2]};
#define PR(f) (int)(off[f + 1] - off[f]), exps + off[f], coefs + off[f], pnorms + off[f], origin + 3 * f
    double v = orc_contr_eri(PR(a), la, PR(b), lb, PR(c), lc, PR(d), ld);
#undef PR
    return norms[a] * norms[b] * norms[c] * norms[d] * v;
}

/* PyQuante/Ints.py:146-167 loop order, 64-bit packed index. */
int orc_get2ints(int64_t nbf, const double *origin, const int64_t *powers, const int64_t *prim_off,
                 const double *exps, const double *coefs, const double *pnorms, const double *norms,
                 double *out)
{
    for (int64_t i = 0; i < nbf; i++)
        for (int64_t j = 0; j <= i; j++) {
            int64_t ij = i * (i + 1) / 2 + j;
            for (int64_t k = 0; k < nbf; k++)
                for (int64_t l = 0; l <= k; l++) {
                    int64_t kl = k * (k + 1) / 2 + l;
                    if (ij <= kl)
                        out[orc_ijkl2intindex(i, j, k, l)] =
                            bf_coulomb(origin, powers, prim_off, exps, coefs, pnorms, norms, i, j, k, l);
                }
        }
    return 0;
}

/* ------------------------------------------------------ 1e integrals --
 * THO formulas (Src/cints.c:190-307), restated; Boys function from above. */
static double fact_d(int n) { double r = 1; for (int i = 2; i <= n; i++) r *= i; return r; }
static double fact2_d(int n) { double r = 1; for (int i = n; i > 1; i -= 2) r *= i; return r; }
static double binom_d(int a, int b) { return fact_d(a) / (fact_d(b) * fact_d(a - b)); }

static double binomial_prefactor(int s, int ia, int ib, double xpa, double xpb)
{
    double sum = 0;
    for (int t = 0; t <= s; t++)
        if (s - ia <= t && t <= ib)
            sum += binom_d(ia, s - t) * binom_d(ib, t) * pow(xpa, ia - s + t) * pow(xpb, ib - t);
    return sum;
}

static double overlap_1d(int l1, int l2, double pax, double pbx, double g)
{
    double s = 0;
    for (int i = 0; i <= (l1 + l2) / 2; i++)
        s += binomial_prefactor(2 * i, l1, l2, pax, pbx) * fact2_d(2 * i - 1) / pow(2 * g, i);
    return s;
}

static double prim_overlap(double a1, const int *l1, const double *A, double a2, const int *l2, const double *B)
{
    double g = a1 + a2, r2 = 0, w = 1;
    for (int i = 0; i < 3; i++) r2 += (A[i] - B[i]) * (A[i] - B[i]);
    for (int i = 0; i < 3; i++) {
        double p = (a1 * A[i] + a2 * B[i]) / g;
        w *= overlap_1d(l1[i], l2[i], p - A[i], p - B[i], g);
    }
    return pow(M_PI / g, 1.5) * exp(-a1 * a2 * r2 / g) * w;
}

static double prim_kinetic(double a1, const int *l1, const double *A, double a2, const int *l2, const double *B)
{
    int L2 = l2[0] + l2[1] + l2[2];
    double t0 = a2 * (2 * L2 + 3) * prim_overlap(a1, l1, A, a2, l2, B), t1 = 0, t2 = 0;
    for (int i = 0; i < 3; i++) {
        int lp[3] = {l2[0], l2[1], l2[2]};
        lp[i] += 2;
        t1 += prim_overlap(a1, l1, A, a2, lp, B);
        if (l2[i] >= 2) {
            int lm[3] = {l2[0], l2[1], l2[2]};
            lm[i] -= 2;
            t2 += l2[i] * (l2[i] - 1) * prim_overlap(a1, l1, A, a2, lm, B);
        }
    }
    return t0 - 2 * a2 * a2 * t1 - 0.5 * t2;
}

static void a_array(int l1, int l2, double pa, double pb, double cp, double g, double *Aout)
{
    int imax = l1 + l2 + 1;
    for (int i = 0; i < imax; i++) Aout[i] = 0;
    for (int i = 0; i < imax; i++)
        for (int r = 0; r <= i / 2; r++)
            for (int u = 0; u <= (i - 2 * r) / 2; u++) {
                int I = i - 2 * r - u;
                Aout[I] += ((i & 1) ? -1.0 : 1.0) * binomial_prefactor(i, l1, l2, pa, pb) * ((u & 1) ? -1.0 : 1.0) *
                           fact_d(i) * pow(cp, i - 2 * r - 2 * u) * pow(0.25 / g, r + u) /
                           (fact_d(r) * fact_d(u) * fact_d(i - 2 * r - 2 * u));
            }
}

static double prim_nuclear(double a1, const int *l1, const double *A, double a2, const int *l2, const double *B,
                           const double *Cn)
{
    double g = a1 + a2, P[3], rab2 = 0, rcp2 = 0, Ax[16], Ay[16], Az[16];
    for (int i = 0; i < 3; i++) {
        P[i] = (a1 * A[i] + a2 * B[i]) / g;
        rab2 += (A[i] - B[i]) * (A[i] - B[i]);
        rcp2 += (Cn[i] - P[i]) * (Cn[i] - P[i]);
    }
    a_array(l1[0], l2[0], P[0] - A[0], P[0] - B[0], P[0] - Cn[0], g, Ax);
    a_array(l1[1], l2[1], P[1] - A[1], P[1] - B[1], P[1] - Cn[1], g, Ay);
    a_array(l1[2], l2[2], P[2] - A[2], P[2] - B[2], P[2] - Cn[2], g, Az);
    double s = 0;
    for (int I = 0; I <= l1[0] + l2[0]; I++)
        for (int J = 0; J <= l1[1] + l2[1]; J++)
            for (int K = 0; K <= l1[2] + l2[2]; K++) s += Ax[I] * Ay[J] * Az[K] * orc_boys(I + J + K, rcp2 * g);
    return -2 * M_PI / g * exp(-a1 * a2 * rab2 / g) * s;
}

/* PyQuante/Ints.py:73-87: S = CGBF.overlap, h = CGBF.kinetic + sum_atoms Z CGBF.nuclear */
void orc_get1ints(int64_t nbf, const double *origin, const int64_t *powers, const int64_t *off,
                  const double *exps, const double *coefs, const double *pnorms, const double *norms,
                  int64_t natoms, const double *atom_xyz, const double *atom_z, double *S, double *h)
{
    for (int64_t i = 0; i < nbf; i++)
        for (int64_t j = 0; j < nbf; j++) {
            int li[3] = {(int)powers[3 * i], (int)powers[3 * i + 1], (int)powers[3 * i + 2]};
            int lj[3] = {(int)powers[3 * j], (int)powers[3 * j + 1], (int)powers[3 * j + 2]};
            double s = 0, t = 0, v = 0;
            for (int64_t p = off[i]; p < off[i + 1]; p++)
                for (int64_t q = off[j]; q < off[j + 1]; q++) {
                    double w = coefs[p] * coefs[q] * pnorms[p] * pnorms[q];
                    s += w * prim_overlap(exps[p], li, origin + 3 * i, exps[q], lj, origin + 3 * j);
                    t += w * prim_kinetic(exps[p], li, origin + 3 * i, exps[q], lj, origin + 3 * j);
                    for (int64_t a = 0; a < natoms; a++)
                        v += atom_z[a] * w *
                             prim_nuclear(exps[p], li, origin + 3 * i, exps[q], lj, origin + 3 * j, atom_xyz + 3 * a);
                }
            S[i * nbf + j] = norms[i] * norms[j] * s;
            h[i * nbf + j] = norms[i] * norms[j] * (t + v);
        }
}

/* PyQuante/Ints.py:195-223: J_ij = sum_kl (ij|kl) D_kl, K_ij = sum_kl (ik|jl) D_kl. */
void orc_getJK(int64_t nbf, const double *ints, const double *D, double *J, double *K)
{
    for (int64_t i = 0; i < nbf; i++)
        for (int64_t j = 0; j <= i; j++) {
            double sj = 0, sk = 0;
            for (int64_t k = 0; k < nbf; k++)
                for (int64_t l = 0; l < nbf; l++) {
                    sj += ints[orc_ijkl2intindex(i, j, k, l)] * D[k * nbf + l];
                    sk += ints[orc_ijkl2intindex(i, k, j, l)] * D[k * nbf + l];
                }
            J[i * nbf + j] = J[j * nbf + i] = sj;
            K[i * nbf + j] = K[j * nbf + i] = sk;
        }
}
