// Device building blocks shared by every kernel of the engine:
//   - the Boys function F_m(T) (table + 8-term Taylor + downward recursion),
//   - Rys roots/weights (piecewise Chebyshev tables, large-T limit),
//   - cartesian-component helpers in PyQuante's order (PyQuante/Ints.py:23-29),
//   - the 2-D Rys recurrence and the horizontal transfer that together replace
//     Recur/Shift of the reference (Src/crys.c:1481-1534).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "pqb_types.h"

#ifndef PQB_TABQ
#define PQB_TABQ static __device__ const
#endif
#ifndef PQB_CTABQ
#define PQB_CTABQ static __constant__ const
#endif
#include "rys_tables.inc"
#include "boys_top.inc"

namespace pqb {

constexpr double kPi = 3.14159265358979323846;
// sqrt(2) * pi^(5/4): K_ab = sqrt(2) pi^(5/4)/zeta exp(-mu R^2) so that
// K_ab K_cd / sqrt(zeta+eta) = 2 pi^(5/2)/(zeta eta sqrt(zeta+eta)) exp(...)
constexpr double kPairPre = 5.9149671727956128778;

// ---------------------------------------------- reciprocal and 1/sqrt --
// Refinement of the single-precision hardware estimates
// (rcp.approx.ftz.f32 and rsqrt.approx.ftz.f32, relative error < 2^-22) by
// one step of the third-order Householder iteration, i.e. the truncated
// series of (1 - e)^(-1) and (1 - e)^(-1/2) in the residual e:
//   1/x:       e = 1 - x r,    r' = r (1 + e + e^2)        (error ~ e^3 ~ 2^-66)
//   1/sqrt(x): e = 1 - x y^2,  y' = y (1 + e/2 + 3 e^2/8)  (error ~ 5 e^3/16)
// Both end within a couple of ulps of the exact value.  x must be positive;
// outside the single-precision normal range (about 1e-36 .. 1e36, where the
// estimate of the rounded x would be 0 or inf) the IEEE operation is used
// instead.  The callers here pass exponent sums, Boys values and Rys
// discriminants, which stay inside it, so that branch is never taken on the
// Fock-build path.
__device__ __forceinline__ double rcp_nr(double x)
{
    const float xf = (float)x;
    if (!(fabsf(xf) > 1e-36f && fabsf(xf) < 1e36f)) return 1.0 / x;
    float rf;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(rf) : "f"(xf));
    const double r = (double)rf;
    const double e = fma(-x, r, 1.0);
    return fma(r, fma(e, e, e), r);
}

__device__ __forceinline__ double rsqrt_nr(double x)
{
    const float xf = (float)x;
    if (!(xf > 1e-36f && xf < 1e36f)) return 1.0 / sqrt(x);
    float yf;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(yf) : "f"(xf));
    const double y = (double)yf;
    const double e = fma(-x * y, y, 1.0);
    return fma(y * e, fma(e, 0.375, 0.5), y);
}

__host__ __device__ constexpr int ncart(int L) { return (L + 1) * (L + 2) / 2; }
// x / y / z exponent of cartesian component i of a shell of angular momentum L,
// PyQuante order (x from L down to 0, then y from L-x down to 0).  With
// n = L - x = number of completed "x levels" before i (closed form for
// L <= 4): x = L - n, z = i - n(n+1)/2, y = n - z.  Plain integer arithmetic
// so unrolled loops fold every index to a constant.
__host__ __device__ constexpr int cart_n(int i) { return (i >= 1) + (i >= 3) + (i >= 6) + (i >= 10); }
__host__ __device__ constexpr int cart_lx(int L, int i) { return L - cart_n(i); }
__host__ __device__ constexpr int cart_lz(int L, int i) { return i - cart_n(i) * (cart_n(i) + 1) / 2; }
__host__ __device__ constexpr int cart_ly(int L, int i) { return cart_n(i) - cart_lz(L, i); }
__host__ __device__ constexpr int cart_l(int L, int i, int axis)
{
    return axis == 0 ? cart_lx(L, i) : (axis == 1 ? cart_ly(L, i) : cart_lz(L, i));
}

// ------------------------------------------------------------------ Boys --
// F_m(T) for m = 0..M into F[].  T < TMAX: F_M by Taylor about the nearest
// grid point T_k = k/16 (|dT| <= 1/32, 8 terms, remainder < 3e-17 F), then
// F_m = (2T F_{m+1} + e^{-T})/(2m+1).  T >= TMAX: F_0 = sqrt(pi/T)/2 and
// F_{m+1} = ((2m+1) F_m - e^{-T})/(2T) (stable for T > m).
template <int M>
__device__ __forceinline__ void boys(double T, double *F)
{
    static_assert(M + 8 <= PQB_BOYS_NORD, "Boys table too short");
    if (T < PQB_BOYS_TMAX) {
        int k = __double2int_rn(T * PQB_BOYS_STEP_INV);
        double d = -(T - k * (1.0 / PQB_BOYS_STEP_INV));
        const double *row = pqb_boys_tab + k * PQB_BOYS_NORD + M;
        double f = __ldg(row + 7);
#pragma unroll
        for (int j = 6; j >= 0; --j) f = fma(f, d * (1.0 / (j + 1)), __ldg(row + j));
        F[M] = f;
        if (M > 0) {
            double e = exp(-T), t2 = 2.0 * T;
#pragma unroll
            for (int m = M - 1; m >= 0; --m) F[m] = fma(t2, F[m + 1], e) * (1.0 / (2 * m + 1));
        }
    } else {
        double it = 1.0 / T;
        F[0] = 0.5 * sqrt(kPi * it);
        if (M > 0) {
            double e = exp(-T), h = 0.5 * it;
#pragma unroll
            for (int m = 0; m < M; ++m) F[m + 1] = ((2 * m + 1) * F[m] - e) * h;
        }
    }
}

// Runtime-order variant (m <= 16) for the general-L kernels.
__device__ __forceinline__ void boys_rt(int M, double T, double *F)
{
    if (T < PQB_BOYS_TMAX) {
        int k = __double2int_rn(T * PQB_BOYS_STEP_INV);
        double d = -(T - k * (1.0 / PQB_BOYS_STEP_INV));
        const double *row = pqb_boys_tab + k * PQB_BOYS_NORD + M;
        double f = __ldg(row + 7);
#pragma unroll
        for (int j = 6; j >= 0; --j) f = fma(f, d * (1.0 / (j + 1)), __ldg(row + j));
        F[M] = f;
        double e = exp(-T), t2 = 2.0 * T;
        for (int m = M - 1; m >= 0; --m) F[m] = fma(t2, F[m + 1], e) / (2 * m + 1);
    } else {
        double it = 1.0 / T, e = exp(-T), h = 0.5 * it;
        F[0] = 0.5 * sqrt(kPi * it);
        for (int m = 0; m < M; ++m) F[m + 1] = ((2 * m + 1) * F[m] - e) * h;
    }
}

// Four doubles from 32-byte aligned global memory with one 256-bit load.
__device__ __forceinline__ void ld4(const double *p, double &a, double &b, double &c, double &d)
{
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];"
        : "=d"(a), "=d"(b), "=d"(c), "=d"(d)
        : "l"(__cvta_generic_to_global(p)));
}

// ------------------------------------------ Boys for the Fock-build kernels --
// F_m(T), m <= 4, from the 16-byte rows {F_top(T_k), exp(-T_k)} of
// boys_top.inc (T_k = k/32, 40-digit values; top = 7 and 10), branch-free
// because the lanes of a warp mix small and large T.
//   T < PQB_BOYSROW_TMAX (40): k = round(32 T), d = T_k - T (|d| <= 1/64);
//     F_j(T_k) for j < top by the downward recursion at T_k,
//     F_j = (2 T_k F_(j+1) + exp(-T_k)) / (2j+1), which keeps or shrinks the
//     relative error of every step; then the Taylor series in d
//     (dF_m/dT = -F_(m+1)), written as nested products
//     sum_j f_j d^j / j! = f_0 + d (f_1 + d/2 (f_2 + ...)):
//       M <= 1: F_0 = P(d) = sum_(j<=7) F_j(T_k) d^j/j! and F_1 = P'(d);
//       M = 3, 4: F_M from F_M .. F_(M+6) at T_k, exp(-T) = exp(-T_k) e^d (7
//       terms), then F_m = (2T F_(m+1) + exp(-T))/(2m+1) downward;
//     truncation below 5e-17 relative.
//   T >= 40: F_0 = sqrt(pi/T)/2 = (sqrt(pi)/2) y with y = 1/sqrt(T) and
//     F_(m+1) = ((2m+1) F_m - exp(-T)) y^2/2.  exp(-T) enters F_m at below
//     2e-12 of its value there, so the hardware single-precision 2^x
//     estimate (ex2.approx, relative error < 2^-22; 0 beyond T = 87, where
//     the term is below 1e-30 of F_m) is exact enough.
// Every lane evaluates both forms (the table row index is clamped) and keeps
// one.  T must be non-negative and below 1e36 (exponent sums times squared
// distances of a molecule).  Against the 40-digit values: below 2e-15
// relative.
__device__ __forceinline__ double rsqrt_nr_unchecked(double x)
{
    float yf;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(yf) : "f"((float)x));
    const double y = (double)yf;
    const double e = fma(-x * y, y, 1.0);
    return fma(y * e, fma(e, 0.375, 0.5), y);
}

__device__ __forceinline__ double exp_neg_estimate(double T)
{
    float r;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"((float)T * -1.44269504088896341f));
    return (double)r;
}

// Two doubles from 16-byte aligned global memory with one 128-bit load.
__device__ __forceinline__ void ld2(const double *p, double &a, double &b)
{
    asm("ld.global.nc.v2.f64 {%0, %1}, [%2];" : "=d"(a), "=d"(b) : "l"(__cvta_generic_to_global(p)));
}

template <int NF>
__device__ __forceinline__ void boys_row1(double T, double *F)
{
    static_assert(NF == 1 || NF == 2, "F_0 or F_0, F_1");
    const bool big = T >= PQB_BOYSROW_TMAX;
    int k = __double2int_rn(T * PQB_BOYSROW_STEP_INV);
    k = k < PQB_BOYSROW_NGRID - 1 ? k : PQB_BOYSROW_NGRID - 1;
    const double Tk = k * (1.0 / PQB_BOYSROW_STEP_INV), d = Tk - T, t2 = 2.0 * Tk;
    double f[8], ek;
    ld2(pqb_boys_top7 + 2 * k, f[7], ek);
#pragma unroll
    for (int j = 6; j >= 0; --j) f[j] = fma(t2, f[j + 1], ek) * (1.0 / (2 * j + 1));
    double dj[7];
#pragma unroll
    for (int j = 0; j < 7; ++j) dj[j] = d * (1.0 / (j + 1));
    double p = f[7], q = f[7];
#pragma unroll
    for (int j = 6; j >= 0; --j) p = fma(p, dj[j], f[j]);
    if (NF > 1) {
#pragma unroll
        for (int j = 5; j >= 0; --j) q = fma(q, dj[j], f[j + 1]);
    }
    const double y = rsqrt_nr_unchecked(T);
    const double a0 = 0.88622692545275801365 * y;
    F[0] = big ? a0 : p;
    if (NF > 1) F[1] = big ? a0 * (0.5 * y * y) : q;
}

template <int M>
__device__ __forceinline__ void boys_rowm(double T, double *F)
{
    static_assert(M == 3 || M == 4, "F_M .. F_(M+6) from F_10");
    const bool big = T >= PQB_BOYSROW_TMAX;
    int k = __double2int_rn(T * PQB_BOYSROW_STEP_INV);
    k = k < PQB_BOYSROW_NGRID - 1 ? k : PQB_BOYSROW_NGRID - 1;
    const double Tk = k * (1.0 / PQB_BOYSROW_STEP_INV), d = Tk - T, tk2 = 2.0 * Tk;
    double f[11], ek;
    ld2(pqb_boys_top10 + 2 * k, f[10], ek);
#pragma unroll
    for (int j = 9; j >= M; --j) f[j] = fma(tk2, f[j + 1], ek) * (1.0 / (2 * j + 1));
    double p = f[M + 6];
#pragma unroll
    for (int j = 5; j >= 0; --j) p = fma(p, d * (1.0 / (j + 1)), f[M + j]);
    double ed = 1.0 / 720.0;
    ed = fma(ed, d, 1.0 / 120.0);
    ed = fma(ed, d, 1.0 / 24.0);
    ed = fma(ed, d, 1.0 / 6.0);
    ed = fma(ed, d, 0.5);
    ed = fma(ed, d, 1.0);
    ed = fma(ed, d, 1.0);
    const double y = rsqrt_nr_unchecked(T), h = 0.5 * y * y;
    const double e = big ? exp_neg_estimate(T) : ek * ed, t2 = 2.0 * T;
    double Ft[M + 1], Fa[M + 1];
    Ft[M] = p;
#pragma unroll
    for (int m = M - 1; m >= 0; --m) Ft[m] = fma(t2, Ft[m + 1], e) * (1.0 / (2 * m + 1));
    Fa[0] = 0.88622692545275801365 * y;
#pragma unroll
    for (int m = 0; m < M; ++m) Fa[m + 1] = ((2 * m + 1) * Fa[m] - e) * h;
#pragma unroll
    for (int m = 0; m <= M; ++m) F[m] = big ? Fa[m] : Ft[m];
}

// F_m(T), m = 0..M for M = 1, 3 or 4.
template <int M>
__device__ __forceinline__ void boys_row(double T, double *F)
{
    if constexpr (M == 1)
        boys_row1<2>(T, F);
    else
        boys_rowm<M>(T, F);
}

// F_0 .. F_LT for the Obara--Saika classes (LT = LA+LB+LC+LD <= 4).
template <int LT>
__device__ __forceinline__ void boys_os(double T, double *F)
{
    static_assert(LT <= 4, "up to F_4");
    if constexpr (LT <= 1) {
        boys_row1<LT + 1>(T, F);
    } else if constexpr (LT <= 3) {
        double G[4];
        boys_rowm<3>(T, G);
#pragma unroll
        for (int m = 0; m <= LT; ++m) F[m] = G[m];
    } else {
        boys_rowm<4>(T, F);
    }
}

// ------------------------------------------------ single precision (mixed) --
// The FP32 kernels of the mixed mode evaluate the Boys function and the Rys
// rules in single precision.

// Eight floats from 32-byte aligned global memory with one 256-bit load.
__device__ __forceinline__ void ld8f(const float *p, float *r)
{
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(r[0]), "=f"(r[1]), "=f"(r[2]), "=f"(r[3]), "=f"(r[4]), "=f"(r[5]), "=f"(r[6]), "=f"(r[7])
        : "l"(__cvta_generic_to_global(p)));
}

// F_0 .. F_LT in single precision for the Obara--Saika classes, from the
// 8-byte rows {F_7(T_k), exp(-T_k)} (pqb_boys_top7_f32), branch-free like
// boys_os: F_j(T_k) by the downward recursion, Taylor
// series of degree 4 (F_0, F_1) or 3 (F_M, M = 3, 4) and a 4-term e^d, then
// the downward recursion at T; for T >= 40 the large-T forms in single
// precision (rsqrtf; exp(-T) from ex2.approx).  Truncation below 2e-9
// relative.
__device__ __forceinline__ void ld2f(const float *p, float &a, float &b)
{
    asm("ld.global.nc.v2.f32 {%0, %1}, [%2];" : "=f"(a), "=f"(b) : "l"(__cvta_generic_to_global(p)));
}

template <int LT>
__device__ __forceinline__ void boys_os_f32(float T, float *F)
{
    static_assert(LT <= 4, "up to F_4");
    const bool big = T >= (float)PQB_BOYSROW_TMAX;
    int k = __float2int_rn(T * PQB_BOYSROW_STEP_INV);
    k = k < PQB_BOYSROW_NGRID - 1 ? k : PQB_BOYSROW_NGRID - 1;
    const float Tk = k * (1.0f / PQB_BOYSROW_STEP_INV), d = Tk - T, tk2 = 2.0f * Tk;
    float f[8], ek;
    ld2f(pqb_boys_top7_f32 + 2 * k, f[7], ek);
    const float y = rsqrtf(T), h = 0.5f * y * y, a0 = 0.886226925f * y;
    if constexpr (LT <= 1) {
#pragma unroll
        for (int j = 6; j >= 0; --j) f[j] = fmaf(tk2, f[j + 1], ek) * (1.0f / (2 * j + 1));
        float dj[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) dj[j] = d * (1.0f / (j + 1));
        float p = f[4], q = f[4];
#pragma unroll
        for (int j = 3; j >= 0; --j) p = fmaf(p, dj[j], f[j]);
#pragma unroll
        for (int j = 2; j >= 0; --j) q = fmaf(q, dj[j], f[j + 1]);
        F[0] = big ? a0 : p;
        if (LT == 1) F[1] = big ? a0 * h : q;
    } else {
        constexpr int M = LT <= 3 ? 3 : 4;
#pragma unroll
        for (int j = 6; j >= M; --j) f[j] = fmaf(tk2, f[j + 1], ek) * (1.0f / (2 * j + 1));
        float p = f[M + 3];
#pragma unroll
        for (int j = 2; j >= 0; --j) p = fmaf(p, d * (1.0f / (j + 1)), f[M + j]);
        float ed = fmaf(d, 1.0f / 6.0f, 0.5f);
        ed = fmaf(ed, d, 1.0f);
        ed = fmaf(ed, d, 1.0f);
        float ebig;
        asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(ebig) : "f"(T * -1.44269504f));
        const float e = big ? ebig : ek * ed, t2 = 2.0f * T;
        float Ft[M + 1], Fa[M + 1];
        Ft[M] = p;
#pragma unroll
        for (int m = M - 1; m >= 0; --m) Ft[m] = fmaf(t2, Ft[m + 1], e) * (1.0f / (2 * m + 1));
        Fa[0] = a0;
#pragma unroll
        for (int m = 0; m < M; ++m) Fa[m + 1] = ((2 * m + 1) * Fa[m] - e) * h;
#pragma unroll
        for (int m = 0; m <= LT; ++m) F[m] = big ? Fa[m] : Ft[m];
    }
}

// Root r of the n-point rule at T < pqb_rys_tasym[n] from the single-precision
// Chebyshev table (7 coefficient pairs, interleaved, per (n, interval, root):
// two 256-bit loads).
__device__ __forceinline__ void rys_root_f32(int n, int r, float T, float &u, float &w)
{
    const int iv = (int)T;
    const float x = 2.0f * (T - iv) - 1.0f, x2 = 2.0f * x;
    const float *c = pqb_rys_coef_f32 + (pqb_rys_offset[n] / (2 * PQB_RYS_NCOEF) + iv * n + r) * 16;
    float cc[16];
    ld8f(c, cc);
    ld8f(c + 8, cc + 8);
    float bu1 = 0.0f, bu2 = 0.0f, bw1 = 0.0f, bw2 = 0.0f;
#pragma unroll
    for (int k = PQB_RYS_NCOEF_F32 - 1; k >= 1; --k) {
        const float tu = fmaf(x2, bu1, cc[2 * k] - bu2), tw = fmaf(x2, bw1, cc[2 * k + 1] - bw2);
        bu2 = bu1;
        bu1 = tu;
        bw2 = bw1;
        bw1 = tw;
    }
    u = fmaf(x, bu1, cc[0] - bu2);
    w = fmaf(x, bw1, cc[1] - bw2);
}

// All NR roots at T (single precision): moments of a Boys row for NR <= 2,
// the truncated Chebyshev table for NR >= 3; FP64 large-T forms above the
// tables (PQB_BOYSROW_TMAX for the Boys rows, pqb_rys_tasym[NR] otherwise).
template <int NR>
__device__ __forceinline__ void rys_roots_f32(float T, float *u, float *w)
{
    const bool large = NR <= 2 ? T >= (float)PQB_BOYSROW_TMAX : T >= (float)pqb_rys_tasym[NR];
    if (large) {
        const double Td = (double)T, it = rcp_nr(Td), rit = rsqrt_nr(Td);
        if constexpr (NR <= 2) {
            // F_m for the moments, exact large-T forms in FP64
            double F[4];
            F[0] = 0.88622692545275801365 * rit;
            const double e = exp(-Td), h = 0.5 * it;
#pragma unroll
            for (int m = 0; m < 2 * NR - 1; ++m) F[m + 1] = ((2 * m + 1) * F[m] - e) * h;
            if constexpr (NR == 1) {
                w[0] = (float)F[0];
                u[0] = (float)(F[1] * rcp_nr(F[0]));
            } else {
                const double id = rcp_nr(fma(F[0], F[2], -F[1] * F[1]));
                const double a1 = fma(F[1], F[2], -F[0] * F[3]) * id, a0 = fma(F[1], F[3], -F[2] * F[2]) * id;
                const double disc = fma(a1, a1, -4.0 * a0), rs = rsqrt_nr(disc);
                const double ub = 0.5 * fma(disc, rs, -a1);
                u[0] = (float)(a0 * rcp_nr(ub));
                u[1] = (float)ub;
                const double w0 = fma(ub, F[0], -F[1]) * rs;
                w[0] = (float)w0;
                w[1] = (float)(F[0] - w0);
            }
        } else {
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                u[r] = (float)(pqb_rys_asym_root[NR][r] * it);
                w[r] = (float)(pqb_rys_asym_weight[NR][r] * rit);
            }
        }
        return;
    }
    if constexpr (NR == 1) {
        float F[2];
        boys_os_f32<1>(T, F);
        w[0] = F[0];
        u[0] = __fdividef(F[1], F[0]);
    } else if constexpr (NR == 2) {
        float F[4];
        boys_os_f32<3>(T, F);
        const float id = __fdividef(1.0f, fmaf(F[0], F[2], -F[1] * F[1]));
        const float a1 = fmaf(F[1], F[2], -F[0] * F[3]) * id, a0 = fmaf(F[1], F[3], -F[2] * F[2]) * id;
        const float disc = fmaf(a1, a1, -4.0f * a0), rs = rsqrtf(disc);
        const float ub = 0.5f * fmaf(disc, rs, -a1);
        u[0] = __fdividef(a0, ub);
        u[1] = ub;
        w[0] = fmaf(ub, F[0], -F[1]) * rs;
        w[1] = F[0] - w[0];
    } else {
#pragma unroll
        for (int r = 0; r < NR; ++r) rys_root_f32(NR, r, T, u[r], w[r]);
    }
}

// ------------------------------------------------------------------- Rys --
// Root r (0-based, ascending) of the n-point Rys rule at T, as u = t^2 in
// (0,1), and its weight (sum_r w_r = F_0(T)).  Below the large-T limit both
// come from degree-13 Chebyshev series on the unit interval of T holding it;
// the table row of (n, interval, root) holds the 14 coefficient pairs
// (root_k, weight_k) interleaved, read with seven 256-bit loads, and the two
// Clenshaw recurrences run side by side.
__device__ __forceinline__ void rys_root(int n, int r, double T, double &u, double &w)
{
    static_assert(PQB_RYS_NCOEF == 14, "seven 256-bit loads per root");
    if (T < pqb_rys_tasym[n]) {
        const int iv = (int)T;
        const double x = 2.0 * (T - iv) - 1.0, x2 = 2.0 * x;
        const double *c = pqb_rys_coef + pqb_rys_offset[n] + (iv * n + r) * (2 * PQB_RYS_NCOEF);
        double cu[PQB_RYS_NCOEF], cw[PQB_RYS_NCOEF];
#pragma unroll
        for (int j = 0; j < PQB_RYS_NCOEF / 2; ++j) ld4(c + 4 * j, cu[2 * j], cw[2 * j], cu[2 * j + 1], cw[2 * j + 1]);
        double bu1 = 0.0, bu2 = 0.0, bw1 = 0.0, bw2 = 0.0;
#pragma unroll
        for (int k = PQB_RYS_NCOEF - 1; k >= 1; --k) {
            const double tu = fma(x2, bu1, cu[k] - bu2), tw = fma(x2, bw1, cw[k] - bw2);
            bu2 = bu1;
            bu1 = tu;
            bw2 = bw1;
            bw1 = tw;
        }
        u = fma(x, bu1, cu[0] - bu2);
        w = fma(x, bw1, cw[0] - bw2);
    } else {
        const double it = 1.0 / T;
        u = pqb_rys_asym_root[n][r] * it;
        w = pqb_rys_asym_weight[n][r] * sqrt(it);
    }
}

// All NR roots at T.  One root (total angular momentum <= 1) comes straight
// from the Boys function: u = F_1/F_0, w = F_0 (8 table loads instead of 28).
template <int NR>
__device__ __forceinline__ void rys_roots(double T, double *u, double *w)
{
    if constexpr (NR == 1) {
        double F[2];
        boys<1>(T, F);
        w[0] = F[0];
        u[0] = F[1] / F[0];
    } else {
#pragma unroll
        for (int r = 0; r < NR; ++r) rys_root(NR, r, T, u[r], w[r]);
    }
}

// All NR roots at T for the integral kernels.  NR = 1 and NR = 2 come from
// one compact Boys row (boys_row): the n-point rule is the Gauss rule of the moments
// F_0..F_(2n-1)(T) (sum_r w_r u_r^k = F_k), so
//   n = 1:  u = F1/F0, w = F0;
//   n = 2:  the monic orthogonal polynomial u^2 + a1 u + a0 solves
//           F2 + a1 F1 + a0 F0 = 0, F3 + a1 F2 + a0 F1 = 0; its larger root
//           u_b = (-a1 + s)/2 (s^2 = a1^2 - 4 a0), the smaller u_s = a0/u_b,
//           and w_s = (u_b F0 - F1)/s, w_b = F0 - w_s.
// This 2x2 moment problem is well conditioned for every T (checked against
// 40-digit Golub--Welsch rules: 3e-15 relative), and costs one table row and
// an exp instead of 4 Chebyshev series.  NR >= 3 uses the tables.
template <int NR>
__device__ __forceinline__ void rys_roots_fast(double T, double *u, double *w)
{
    if constexpr (NR == 1) {
        double F[2];
        boys_row<1>(T, F);
        w[0] = F[0];
        u[0] = F[1] * rcp_nr(F[0]);
    } else if constexpr (NR == 2) {
        double F[4];
        boys_row<3>(T, F);
        const double id = rcp_nr(fma(F[0], F[2], -F[1] * F[1]));
        const double a1 = fma(F[1], F[2], -F[0] * F[3]) * id;
        const double a0 = fma(F[1], F[3], -F[2] * F[2]) * id;
        const double disc = fma(a1, a1, -4.0 * a0);
        const double rs = rsqrt_nr(disc);
        const double ub = 0.5 * fma(disc, rs, -a1);
        u[0] = a0 * rcp_nr(ub);
        u[1] = ub;
        w[0] = fma(ub, F[0], -F[1]) * rs;
        w[1] = F[0] - w[0];
    } else {
#pragma unroll
        for (int r = 0; r < NR; ++r) rys_root(NR, r, T, u[r], w[r]);
    }
}

// Per-root coefficients of the 2-D recurrence (no divisions: izeta, ieta and
// izpe = 1/(zeta+eta) come precomputed):
//   b00 = u/(2(zeta+eta)),  b10 = (1 - eta u/(zeta+eta))/(2 zeta),
//   b01 = (1 - zeta u/(zeta+eta))/(2 eta),
//   c00 = PA - ce PQ, c01 = QC + cz PQ with ce = eta u/(zeta+eta), cz = zeta u/(zeta+eta).
struct RysCoef {
    double b00, b10, b01, ce, cz;
};

__device__ __forceinline__ RysCoef rys_coef(double u, double zeta, double eta, double izeta, double ieta,
                                            double izpe)
{
    const double ue = u * izpe;
    RysCoef k;
    k.b00 = 0.5 * ue;
    k.ce = eta * ue;
    k.cz = zeta * ue;
    k.b10 = 0.5 * izeta * (1.0 - k.ce);
    k.b01 = 0.5 * ieta * (1.0 - k.cz);
    return k;
}

// ------------------------------------------------ 2-D Rys integrals (one axis)
// For one root u and one cartesian axis: G(n,m) = I_x(n,0|m,0) by the Rys
// recurrence (bra exponent sum zeta, ket eta), then the horizontal transfer
// I(a,b+1|c,d) = I(a+1,b|c,d) + AB I(a,b|c,d) and likewise on the ket, giving
// out[((a*(LB+1)+b)*(LC+1)+c)*(LD+1)+d] for a<=LA, b<=LB, c<=LC, d<=LD.
// `scale` multiplies every output (the root weight times the quartet
// prefactor goes on one axis).  All sizes are compile-time: fully unrolled,
// register resident.
template <int LA, int LB, int LC, int LD, typename R>
__device__ __forceinline__ void rys2d_c(const RysCoef &k, double PA, double QC, double PQ, double AB, double CD,
                                        double scale, R *out)
{
    constexpr int NB = LA + LB, MK = LC + LD;
    const double b00 = k.b00, b10 = k.b10, b01 = k.b01;
    const double c00 = fma(-k.ce, PQ, PA);
    const double c01 = fma(k.cz, PQ, QC);
    R g[NB + 1][MK + 1];
    g[0][0] = (R)scale;
    if (NB > 0) g[1][0] = (R)(c00 * scale);
#pragma unroll
    for (int n = 1; n < NB; ++n) g[n + 1][0] = (R)(n * b10) * g[n - 1][0] + (R)c00 * g[n][0];
#pragma unroll
    for (int n = 0; n <= NB; ++n) {
        if (MK > 0) g[n][1] = (R)c01 * g[n][0] + (n > 0 ? (R)(n * b00) * g[n - 1][0] : (R)0);
#pragma unroll
        for (int m = 1; m < MK; ++m)
            g[n][m + 1] = (R)(m * b01) * g[n][m - 1] + (R)c01 * g[n][m] +
                          (n > 0 ? (R)(n * b00) * g[n - 1][m] : (R)0);
    }
    // ket transfer: h[n][c][d] for n <= NB, c <= LC, d <= LD
    R h[NB + 1][LC + 1][LD + 1];
#pragma unroll
    for (int n = 0; n <= NB; ++n) {
        R t[MK + 1][LD + 1];
#pragma unroll
        for (int m = 0; m <= MK; ++m) t[m][0] = g[n][m];
#pragma unroll
        for (int d = 1; d <= LD; ++d)
#pragma unroll
            for (int m = 0; m + d <= MK; ++m) t[m][d] = t[m + 1][d - 1] + (R)CD * t[m][d - 1];
#pragma unroll
        for (int c = 0; c <= LC; ++c)
#pragma unroll
            for (int d = 0; d <= LD; ++d) h[n][c][d] = t[c][d];
    }
    // bra transfer
#pragma unroll
    for (int c = 0; c <= LC; ++c)
#pragma unroll
        for (int d = 0; d <= LD; ++d) {
            R t[NB + 1][LB + 1];
#pragma unroll
            for (int n = 0; n <= NB; ++n) t[n][0] = h[n][c][d];
#pragma unroll
            for (int b = 1; b <= LB; ++b)
#pragma unroll
                for (int n = 0; n + b <= NB; ++n) t[n][b] = t[n + 1][b - 1] + (R)AB * t[n][b - 1];
#pragma unroll
            for (int a = 0; a <= LA; ++a)
#pragma unroll
                for (int b = 0; b <= LB; ++b) out[((a * (LB + 1) + b) * (LC + 1) + c) * (LD + 1) + d] = t[a][b];
        }
}

// The 2-D tables in single precision from single-precision inputs (mixed
// mode): the same recurrence and transfers as rys2d_c.
template <int LA, int LB, int LC, int LD>
__device__ __forceinline__ void rys2d_f(float b00, float b10, float b01, float c00, float c01, float AB, float CD,
                                        float scale, float *out)
{
    constexpr int NB = LA + LB, MK = LC + LD;
    float g[NB + 1][MK + 1];
    g[0][0] = scale;
    if (NB > 0) g[1][0] = c00 * scale;
#pragma unroll
    for (int n = 1; n < NB; ++n) g[n + 1][0] = (n * b10) * g[n - 1][0] + c00 * g[n][0];
#pragma unroll
    for (int n = 0; n <= NB; ++n) {
        if (MK > 0) g[n][1] = c01 * g[n][0] + (n > 0 ? (n * b00) * g[n - 1][0] : 0.0f);
#pragma unroll
        for (int m = 1; m < MK; ++m)
            g[n][m + 1] = (m * b01) * g[n][m - 1] + c01 * g[n][m] + (n > 0 ? (n * b00) * g[n - 1][m] : 0.0f);
    }
    float h[NB + 1][LC + 1][LD + 1];
#pragma unroll
    for (int n = 0; n <= NB; ++n) {
        float t[MK + 1][LD + 1];
#pragma unroll
        for (int m = 0; m <= MK; ++m) t[m][0] = g[n][m];
#pragma unroll
        for (int d = 1; d <= LD; ++d)
#pragma unroll
            for (int m = 0; m + d <= MK; ++m) t[m][d] = t[m + 1][d - 1] + CD * t[m][d - 1];
#pragma unroll
        for (int c = 0; c <= LC; ++c)
#pragma unroll
            for (int d = 0; d <= LD; ++d) h[n][c][d] = t[c][d];
    }
#pragma unroll
    for (int c = 0; c <= LC; ++c)
#pragma unroll
        for (int d = 0; d <= LD; ++d) {
            float t[NB + 1][LB + 1];
#pragma unroll
            for (int n = 0; n <= NB; ++n) t[n][0] = h[n][c][d];
#pragma unroll
            for (int b = 1; b <= LB; ++b)
#pragma unroll
                for (int n = 0; n + b <= NB; ++n) t[n][b] = t[n + 1][b - 1] + AB * t[n][b - 1];
#pragma unroll
            for (int a = 0; a <= LA; ++a)
#pragma unroll
                for (int b = 0; b <= LB; ++b) out[((a * (LB + 1) + b) * (LC + 1) + c) * (LD + 1) + d] = t[a][b];
        }
}

// The same from (u, zeta, eta) with the divisions done here (general and
// gradient kernels, which are not on the Fock-build path).
template <int LA, int LB, int LC, int LD, typename R>
__device__ __forceinline__ void rys2d(double u, double zeta, double eta, double PA, double QC, double PQ,
                                      double AB, double CD, double scale, R *out)
{
    const double zpe = zeta + eta;
    RysCoef k;
    k.b00 = 0.5 * u / zpe;
    k.b10 = (0.5 - 0.5 * eta / zpe * u) / zeta;
    k.b01 = (0.5 - 0.5 * zeta / zpe * u) / eta;
    k.ce = eta / zpe * u;
    k.cz = zeta / zpe * u;
    rys2d_c<LA, LB, LC, LD, R>(k, PA, QC, PQ, AB, CD, scale, out);
}

// The Fock-build fields of a PrimPair (zeta, 1/zeta, P, K): one 256-bit and
// one 128-bit load.
struct PrimJK {
    double zeta, izeta, P[3], K;
};

__device__ __forceinline__ PrimJK load_prim_jk(const PrimPair *p)
{
    PrimJK r;
    ld4(reinterpret_cast<const double *>(p), r.zeta, r.izeta, r.P[0], r.P[1]);
    const double2 c = __ldg(reinterpret_cast<const double2 *>(p) + 2);
    r.P[2] = c.x;
    r.K = c.y;
    return r;
}

}  // namespace pqb
