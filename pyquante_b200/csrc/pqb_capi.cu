// C ABI of the engine (declared in include/pyquante_b200.h): context,
// shell/pair tables, quartet planning, and the kernels that are not
// class-templated (general-L scalar ERIs by Rys and by Head-Gordon--Pople,
// one-electron integrals, stored-integral J/K, Boys/Rys probes).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <type_traits>
#include <utility>
#include <vector>

#define PQB_TABQ static __device__ const
#define PQB_CTABQ static __constant__ const
#include "../../include/pyquante_b200.h"
#include "eri_launch.h"
#include "pqb_device.cuh"
#include "pqb_types.h"

using namespace pqb;

// Primitive-quartet chunk for the J/K work items: long contractions
// (up to 1296 primitive quartets for a 6-primitive s shell to the fourth)
// are cut so no thread or block slot runs a long serial chain.  Per class,
// tunable with pqb_set_param(PQB_PARAM_CHUNK) (default 16).
static const int kDefaultChunk = 16;

struct pqb_ctx {
    int device = 0;
    int nsm = 148;
    std::string err;
    // basis
    int nbf = 0, nshell = 0;
    std::vector<int> sh_l, sh_np, sh_off, sh_f0;
    std::vector<double> sh_xyz, pr_exp, pr_coef, fscale_h;
    // device tables
    PairInfo *d_pairs = nullptr;
    PrimPair *d_prims = nullptr;
    double *d_fscale = nullptr;
    // direct J/K digest the shells' common-contraction integrals: the density
    // is pre-scaled element-wise by escale[(i,j)] = r_i r_j (r = fscale) into
    // d_Dscaled, and J, K are scaled by the same factors when symmetrised
    double *d_escale = nullptr, *d_Dscaled = nullptr;
    float *d_Dscaled_f = nullptr;    // single-precision copy for the FP32 lists
    double *d_Dscaled2 = nullptr;    // the second density of pqb_jk_direct2 (allocated on first use)
    float *d_Dscaled2_f = nullptr;
    unsigned long long *d_q2 = nullptr;
    std::vector<PairInfo> pairs;
    std::vector<double> Q;           // Schwarz factors (host)
    bool have_q = false;
    // unscreened lists (packed integrals): per class offset/count into d_full
    int4 *d_full = nullptr;
    int64_t full_off[kNumQuartetClass] = {0}, full_cnt[kNumQuartetClass] = {0};
    // Schwarz (diagonal) list
    int4 *d_diag = nullptr;
    int64_t diag_off[kNumQuartetClass] = {0}, diag_cnt[kNumQuartetClass] = {0};
    // screened plan: [0] FP64 part, [1] FP32-eligible part
    int4 *d_plan = nullptr;
    size_t plan_cap = 0;
    int64_t plan_off[2][kNumQuartetClass] = {{0}}, plan_cnt[2][kNumQuartetClass] = {{0}};
    int64_t plan_prims[2][kNumQuartetClass] = {{0}};
    std::vector<int4> plan_h;        // host copy of the plan (for sharding)
    int *d_shell_atom = nullptr;     // atom index of every shell (gradients)
    int2 *d_pk_tiles = nullptr;      // (i, j0) tiles of the stored-integral J/K kernel
    int pk_tiles_n = 0, pk_tiles_nbf = -1;
    bool packed_simple = false;      // force the one-block-per-row stored J/K kernel (tests)
    // batched bases: molecules own consecutive shells/functions; D/J/K hold
    // one dense nm x nm block per molecule, back to back
    int nmol = 1;
    std::vector<int> mol_f0, mol_n, pair_first;   // per molecule; per pair: first pair of its molecule
    std::vector<long long> mol_off;
    long long dense_len = 0;
    long long *d_mol_off = nullptr;
    int *d_mol_n = nullptr;
    int chunk[kNumQuartetClass];     // primitive-quartet chunk per class
    int nstreams = 8;
    int order = 1;                   // class launch order: 0 by cost, 1 high angular momentum first
    // fork/join streams for concurrent class launches
    static constexpr int kStreams = 16;
    cudaStream_t streams[kStreams] = {nullptr};
    cudaEvent_t ev_fork = nullptr, ev_join[kStreams] = {nullptr};
    bool have_plan = false;
    // pqb_jk_direct replays a captured graph of the class launches (one per
    // mode), accumulating into ctx-owned J/K; rebuilt after any change of
    // basis, plan or launch parameters
    bool use_graph = true;
    int plan_threads = 0;            // host threads of pqb_plan (0: automatic)
    cudaStream_t cap_stream = nullptr;
    // graphs: [mode] for one density, [2 + mode] for two (pqb_jk_direct2),
    // [4 + mode] for J alone
    cudaGraphExec_t graph_exec[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    bool graph_warm[6] = {false, false, false, false, false, false};   // one eager build first (one-time launch setup stays out of the capture)
    double *d_Jacc = nullptr, *d_Kacc = nullptr;
    double *d_Jacc2 = nullptr, *d_Kacc2 = nullptr;   // second density's graph accumulators
    // pqb_get2jmk_host: D in, G out, and J, K of its builds outside the graph
    double *d_hD = nullptr, *d_hG = nullptr, *d_hJ = nullptr, *d_hK = nullptr;
    ItemScreen scr{};                // caller-owned molecule mask / shell density bounds of the direct builds
    double *d_Qpair = nullptr;       // Schwarz factor per pair (device)
    int4 *d_shell_info = nullptr;    // per shell: first function within its molecule, functions, molecule
    // small scratch
    double *d_atoms = nullptr;
    size_t atoms_cap = 0;
};

static int fail(pqb_ctx *ctx, int code, const char *fmt, ...)
{
    if (ctx) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        ctx->err = buf;
    }
    return code;
}

#define PQB_CK(ctx, call)                                                                              \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) return fail(ctx, PQB_E_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

static void free_dev(void *p)
{
    if (p) cudaFree(p);
}

// ===================================================================== kernels

// In-place M = M + M^T (the J/K accumulators hold one triangle's worth of
// each unique contribution; see EpiJK), times S element-wise when S is given.
__global__ void symmetrize_kernel(double *M, int n, const double *__restrict__ S)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t P = (int64_t)n * (n + 1) / 2;
    if (t >= P) return;
    int i = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((int64_t)i * (i + 1) / 2 > t) --i;
    while ((int64_t)(i + 1) * (i + 2) / 2 <= t) ++i;
    int j = (int)(t - (int64_t)i * (i + 1) / 2);
    double s = M[(int64_t)i * n + j] + M[(int64_t)j * n + i];
    if (S) s *= S[(int64_t)i * n + j];
    M[(int64_t)i * n + j] = s;
    M[(int64_t)j * n + i] = s;
}

// dmax[s] = max |D_ij| over the rows i of shell s and the columns j of its
// molecule's block (one warp per shell).
__global__ void shell_dmax_kernel(int nshell, const int4 *__restrict__ info, const long long *__restrict__ mol_off,
                                  const int *__restrict__ mol_n, const double *__restrict__ D, double *__restrict__ dmax)
{
    const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (s >= nshell) return;
    const int4 in = info[s];
    const int nm = mol_n[in.z];
    const double *row = D + mol_off[in.z] + (long long)in.x * nm;
    double m = 0.0;
    for (int r = 0; r < in.y; ++r, row += nm)
        for (int j = lane; j < nm; j += 32) m = fmax(m, fabs(row[j]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) dmax[s] = m;
}

// The graph path's epilogue: J and K (K2 == nullptr: J alone) from their
// accumulators, which are left zeroed for the next replay of the build graph
// (so the graph holds no memset nodes).
__global__ void symmetrize_take_kernel(double *__restrict__ A1, double *__restrict__ M1, double *__restrict__ A2,
                                       double *__restrict__ M2, int n, const double *__restrict__ S)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t P = (int64_t)n * (n + 1) / 2;
    if (t >= P) return;
    int i = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((int64_t)i * (i + 1) / 2 > t) --i;
    while ((int64_t)(i + 1) * (i + 2) / 2 <= t) ++i;
    int j = (int)(t - (int64_t)i * (i + 1) / 2);
    const int64_t ij = (int64_t)i * n + j, ji = (int64_t)j * n + i;
    const double sc = S ? S[ij] : 1.0;
    const double s1 = (A1[ij] + A1[ji]) * sc;
    A1[ij] = 0.0;
    A1[ji] = 0.0;
    M1[ij] = s1;
    M1[ji] = s1;
    if (A2) {
        const double s2 = (A2[ij] + A2[ji]) * sc;
        A2[ij] = 0.0;
        A2[ji] = 0.0;
        M2[ij] = s2;
        M2[ji] = s2;
    }
}

// G = 2J - K straight from the graph's J and K accumulators (scaled and
// symmetrised like symmetrize_take_kernel, which it replaces when the caller
// wants G alone), leaving them zeroed.
__global__ void take_2jmk_kernel(double *__restrict__ A1, double *__restrict__ A2, double *__restrict__ G, int n,
                                 const double *__restrict__ S)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    int64_t P = (int64_t)n * (n + 1) / 2;
    if (t >= P) return;
    int i = (int)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while ((int64_t)i * (i + 1) / 2 > t) --i;
    while ((int64_t)(i + 1) * (i + 2) / 2 <= t) ++i;
    int j = (int)(t - (int64_t)i * (i + 1) / 2);
    const int64_t ij = (int64_t)i * n + j, ji = (int64_t)j * n + i;
    const double sc = S ? S[ij] : 1.0;
    const double g = fma(2.0, A1[ij] + A1[ji], -(A2[ij] + A2[ji])) * sc;
    A1[ij] = 0.0;
    A1[ji] = 0.0;
    A2[ij] = 0.0;
    A2[ji] = 0.0;
    G[ij] = g;
    G[ji] = g;
}

__global__ void combine_2jmk_kernel(const double *__restrict__ J, const double *__restrict__ K, double *__restrict__ G,
                                    int64_t len)
{
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < len; t += (int64_t)gridDim.x * blockDim.x)
        G[t] = fma(2.0, J[t], -K[t]);
}

// Batched form: one CUDA block per molecule block of a block-diagonal layout.
__global__ void symmetrize_blocks_kernel(double *M, const long long *__restrict__ off, const int *__restrict__ nm,
                                         const double *__restrict__ S)
{
    const int m = blockIdx.x, n = nm[m];
    double *B = M + off[m];
    const double *SB = S ? S + off[m] : nullptr;
    for (int t = threadIdx.x; t < n * n; t += blockDim.x) {
        const int i = t / n, j = t - i * n;
        if (j > i) continue;
        double s = B[(int64_t)i * n + j] + B[(int64_t)j * n + i];
        if (SB) s *= SB[(int64_t)i * n + j];
        B[(int64_t)i * n + j] = s;
        B[(int64_t)j * n + i] = s;
    }
}

// Y = X * S element-wise (the pre-scaled density of the direct J/K kernels)
// and its single-precision copy Yf.
__global__ void scale_elements_kernel(const double *__restrict__ X, const double *__restrict__ S, double *__restrict__ Y,
                                      float *__restrict__ Yf, int64_t len)
{
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < len; t += (int64_t)gridDim.x * blockDim.x) {
        const double y = X[t] * S[t];
        Y[t] = y;
        Yf[t] = (float)y;
    }
}

__device__ __forceinline__ double binom_d(int n, int k)
{
    double r = 1.0;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
}

// ---- general-L Rys: one thread per function quartet (crys.contr_coulomb
// semantics, Src/crys.c:34-97; the 2-D recursion of ABD eqs 11-16 and the
// binomial transfer of Src/crys.c:1518-1534, in t^2 form).
__device__ double rys_axis_general(double u, double zeta, double eta, double PA, double QC, double PQ, double AB,
                                   double CD, int la, int lb, int lc, int ld)
{
    const int NB = la + lb, MK = lc + ld;
    double G[10][10];
    const double zpe = zeta + eta;
    const double b00 = 0.5 * u / zpe, b10 = (0.5 - 0.5 * eta / zpe * u) / zeta, b01 = (0.5 - 0.5 * zeta / zpe * u) / eta;
    const double c00 = PA - eta / zpe * u * PQ, c01 = QC + zeta / zpe * u * PQ;
    G[0][0] = 1.0;
    if (NB > 0) G[1][0] = c00;
    for (int n = 1; n < NB; ++n) G[n + 1][0] = n * b10 * G[n - 1][0] + c00 * G[n][0];
    for (int n = 0; n <= NB; ++n) {
        if (MK > 0) G[n][1] = c01 * G[n][0] + (n > 0 ? n * b00 * G[n - 1][0] : 0.0);
        for (int m = 1; m < MK; ++m)
            G[n][m + 1] = m * b01 * G[n][m - 1] + c01 * G[n][m] + (n > 0 ? n * b00 * G[n - 1][m] : 0.0);
    }
    double s = 0.0;
    for (int p = 0; p <= lb; ++p) {
        double sp = 0.0;
        for (int q = 0; q <= ld; ++q) sp += binom_d(ld, q) * pow(CD, ld - q) * G[la + p][lc + q];
        s += binom_d(lb, p) * pow(AB, lb - p) * sp;
    }
    return s;
}

struct FuncTable {
    const double *origin;
    const int *powers;
    const int *prim_off;
    const double *exps, *cn, *norms;
};

__global__ void eri_general_rys_kernel(int nq, const int *__restrict__ quartets, FuncTable ft, double *out)
{
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    int f[4];
    for (int x = 0; x < 4; ++x) f[x] = quartets[4 * q + x];
    int L = 0;
    for (int x = 0; x < 4; ++x) L += ft.powers[3 * f[x]] + ft.powers[3 * f[x] + 1] + ft.powers[3 * f[x] + 2];
    if (L > 9) {   // beyond the 5-root tables (the host rejects these first)
        out[q] = nan("");
        return;
    }
    const int nr = L / 2 + 1;
    const double *A = ft.origin + 3 * f[0], *B = ft.origin + 3 * f[1], *C = ft.origin + 3 * f[2], *D = ft.origin + 3 * f[3];
    double sum = 0.0;
    for (int p = ft.prim_off[f[0]]; p < ft.prim_off[f[0] + 1]; ++p)
        for (int qq = ft.prim_off[f[1]]; qq < ft.prim_off[f[1] + 1]; ++qq) {
            const double a = ft.exps[p], b = ft.exps[qq], zeta = a + b;
            double P[3], rab2 = 0.0;
            for (int x = 0; x < 3; ++x) {
                P[x] = (a * A[x] + b * B[x]) / zeta;
                rab2 += (A[x] - B[x]) * (A[x] - B[x]);
            }
            const double Kab = ft.cn[p] * ft.cn[qq] * kPairPre / zeta * exp(-a * b / zeta * rab2);
            for (int r = ft.prim_off[f[2]]; r < ft.prim_off[f[2] + 1]; ++r)
                for (int s = ft.prim_off[f[3]]; s < ft.prim_off[f[3] + 1]; ++s) {
                    const double c = ft.exps[r], d = ft.exps[s], eta = c + d;
                    double Qc[3], rcd2 = 0.0, rpq2 = 0.0;
                    for (int x = 0; x < 3; ++x) {
                        Qc[x] = (c * C[x] + d * D[x]) / eta;
                        rcd2 += (C[x] - D[x]) * (C[x] - D[x]);
                        rpq2 += (P[x] - Qc[x]) * (P[x] - Qc[x]);
                    }
                    const double Kcd = ft.cn[r] * ft.cn[s] * kPairPre / eta * exp(-c * d / eta * rcd2);
                    const double T = zeta * eta / (zeta + eta) * rpq2;
                    const double pre = Kab * Kcd / sqrt(zeta + eta);
                    for (int k = 0; k < nr; ++k) {
                        double u, w;
                        rys_root(nr, k, T, u, w);
                        double prod = w * pre;
                        for (int x = 0; x < 3; ++x)
                            prod *= rys_axis_general(u, zeta, eta, P[x] - A[x], Qc[x] - C[x], P[x] - Qc[x], A[x] - B[x],
                                                     C[x] - D[x], ft.powers[3 * f[0] + x], ft.powers[3 * f[1] + x],
                                                     ft.powers[3 * f[2] + x], ft.powers[3 * f[3] + x]);
                        sum += prod;
                    }
                }
        }
    out[q] = ft.norms[f[0]] * ft.norms[f[1]] * ft.norms[f[2]] * ft.norms[f[3]] * sum;
}

// ---- general-L Head-Gordon--Pople (the scheme of Src/chgp.c:78-419): an
// Obara--Saika VRR for (e0|f0)^(m), computed bottom-up over the box
// e' <= a+b, f' <= c+d (componentwise), then the HRR
// (a,b+1_i|..) = (a+1_i,b|..) + AB_i (a,b|..) applied in closed (binomial)
// form.  Boys values by table + downward recursion.  Per-side momentum
// |a|+|b| <= 4 and |c|+|d| <= 4 bound the box to 12 x 12 entries.
#define PQB_HGP_BOX 12
__global__ void eri_general_hgp_kernel(int nq, int aux_m, const int *__restrict__ quartets, FuncTable ft, double *out)
{
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nq) return;
    int f[4];
    for (int x = 0; x < 4; ++x) f[x] = quartets[4 * q + x];
    int la[3], lb[3], lc[3], ld[3], E[3], F[3];
    for (int x = 0; x < 3; ++x) {
        la[x] = ft.powers[3 * f[0] + x];
        lb[x] = ft.powers[3 * f[1] + x];
        lc[x] = ft.powers[3 * f[2] + x];
        ld[x] = ft.powers[3 * f[3] + x];
        E[x] = la[x] + lb[x];
        F[x] = lc[x] + ld[x];
    }
    const int Es[3] = {1, E[0] + 1, (E[0] + 1) * (E[1] + 1)};
    const int Fs[3] = {1, F[0] + 1, (F[0] + 1) * (F[1] + 1)};
    const int nE = (E[0] + 1) * (E[1] + 1) * (E[2] + 1), nF = (F[0] + 1) * (F[1] + 1) * (F[2] + 1);
    const int M = E[0] + E[1] + E[2] + F[0] + F[1] + F[2] + aux_m;
    if (nE > PQB_HGP_BOX || nF > PQB_HGP_BOX || M > 8 || aux_m < 0) {   // outside the box (the host rejects these first)
        out[q] = nan("");
        return;
    }
    double V[PQB_HGP_BOX * PQB_HGP_BOX * 9];   // [e][f][m], m <= 8
    const double *A = ft.origin + 3 * f[0], *B = ft.origin + 3 * f[1], *C = ft.origin + 3 * f[2], *D = ft.origin + 3 * f[3];
    double sum = 0.0;
    for (int p = ft.prim_off[f[0]]; p < ft.prim_off[f[0] + 1]; ++p)
        for (int p2 = ft.prim_off[f[1]]; p2 < ft.prim_off[f[1] + 1]; ++p2)
            for (int r = ft.prim_off[f[2]]; r < ft.prim_off[f[2] + 1]; ++r)
                for (int s = ft.prim_off[f[3]]; s < ft.prim_off[f[3] + 1]; ++s) {
                    const double a = ft.exps[p], b = ft.exps[p2], c = ft.exps[r], d = ft.exps[s];
                    const double zeta = a + b, eta = c + d, ze = zeta + eta;
                    double PA[3], QC[3], WP[3], WQ[3], rab2 = 0, rcd2 = 0, rpq2 = 0;
                    for (int x = 0; x < 3; ++x) {
                        const double P = (a * A[x] + b * B[x]) / zeta, Qx = (c * C[x] + d * D[x]) / eta;
                        const double W = (zeta * P + eta * Qx) / ze;
                        PA[x] = P - A[x];
                        QC[x] = Qx - C[x];
                        WP[x] = W - P;
                        WQ[x] = W - Qx;
                        rab2 += (A[x] - B[x]) * (A[x] - B[x]);
                        rcd2 += (C[x] - D[x]) * (C[x] - D[x]);
                        rpq2 += (P - Qx) * (P - Qx);
                    }
                    const double pre = ft.cn[p] * ft.cn[p2] * ft.cn[r] * ft.cn[s] * 2.0 * pow(kPi, 2.5) /
                                       (zeta * eta * sqrt(ze)) * exp(-a * b / zeta * rab2 - c * d / eta * rcd2);
                    double Fm[17];
                    boys_rt(M, zeta * eta / ze * rpq2, Fm);
                    const double o2z = 0.5 / zeta, o2e = 0.5 / eta, o2ze = 0.5 / ze, rz = eta / ze, re = zeta / ze;
                    for (int ex = 0; ex <= E[0]; ++ex)
                        for (int ey = 0; ey <= E[1]; ++ey)
                            for (int ez = 0; ez <= E[2]; ++ez)
                                for (int fx = 0; fx <= F[0]; ++fx)
                                    for (int fy = 0; fy <= F[1]; ++fy)
                                        for (int fz = 0; fz <= F[2]; ++fz) {
                                            const int e3[3] = {ex, ey, ez}, f3[3] = {fx, fy, fz};
                                            const int ie = ex * Es[0] + ey * Es[1] + ez * Es[2];
                                            const int jf = fx * Fs[0] + fy * Fs[1] + fz * Fs[2];
                                            const int tot = ex + ey + ez + fx + fy + fz;
                                            for (int m = 0; m <= M - tot; ++m) {
                                                double v;
                                                if (ex + ey + ez > 0) {
                                                    const int i = ex ? 0 : (ey ? 1 : 2);
                                                    const int e1 = ie - Es[i];
                                                    v = PA[i] * V[(e1 * nF + jf) * 9 + m] + WP[i] * V[(e1 * nF + jf) * 9 + m + 1];
                                                    if (e3[i] > 1) {
                                                        const int e2 = e1 - Es[i];
                                                        v += (e3[i] - 1) * o2z *
                                                             (V[(e2 * nF + jf) * 9 + m] - rz * V[(e2 * nF + jf) * 9 + m + 1]);
                                                    }
                                                    if (f3[i] > 0) v += f3[i] * o2ze * V[(e1 * nF + jf - Fs[i]) * 9 + m + 1];
                                                } else if (fx + fy + fz > 0) {
                                                    const int i = fx ? 0 : (fy ? 1 : 2);
                                                    const int f1 = jf - Fs[i];
                                                    v = QC[i] * V[(ie * nF + f1) * 9 + m] + WQ[i] * V[(ie * nF + f1) * 9 + m + 1];
                                                    if (f3[i] > 1) {
                                                        const int f2 = f1 - Fs[i];
                                                        v += (f3[i] - 1) * o2e *
                                                             (V[(ie * nF + f2) * 9 + m] - re * V[(ie * nF + f2) * 9 + m + 1]);
                                                    }
                                                } else {
                                                    v = pre * Fm[m];
                                                }
                                                V[(ie * nF + jf) * 9 + m] = v;
                                            }
                                        }
                    (void)nE;
                    // HRR in binomial form: b onto a, d onto c
                    double s2 = 0.0;
                    for (int bx = 0; bx <= lb[0]; ++bx)
                        for (int by = 0; by <= lb[1]; ++by)
                            for (int bz = 0; bz <= lb[2]; ++bz) {
                                const double cb = binom_d(lb[0], bx) * binom_d(lb[1], by) * binom_d(lb[2], bz) *
                                                  pow(A[0] - B[0], lb[0] - bx) * pow(A[1] - B[1], lb[1] - by) *
                                                  pow(A[2] - B[2], lb[2] - bz);
                                const int ie = (la[0] + bx) * Es[0] + (la[1] + by) * Es[1] + (la[2] + bz) * Es[2];
                                for (int dx = 0; dx <= ld[0]; ++dx)
                                    for (int dy = 0; dy <= ld[1]; ++dy)
                                        for (int dz = 0; dz <= ld[2]; ++dz) {
                                            const double cdf = binom_d(ld[0], dx) * binom_d(ld[1], dy) *
                                                               binom_d(ld[2], dz) * pow(C[0] - D[0], ld[0] - dx) *
                                                               pow(C[1] - D[1], ld[1] - dy) * pow(C[2] - D[2], ld[2] - dz);
                                            const int jf =
                                                (lc[0] + dx) * Fs[0] + (lc[1] + dy) * Fs[1] + (lc[2] + dz) * Fs[2];
                                            s2 += cb * cdf * V[(ie * nF + jf) * 9 + aux_m];
                                        }
                            }
                    sum += s2;
                }
    out[q] = ft.norms[f[0]] * ft.norms[f[1]] * ft.norms[f[2]] * ft.norms[f[3]] * sum;
}

// ---- one-electron integrals, one thread per (i, j): overlap and kinetic by
// the Obara--Saika 1-D overlap recursion (the kinetic combination of
// Src/cints.c:190-213), nuclear attraction by 1-electron Rys quadrature
// (T = zeta |P-C|^2, n = (li+lj)/2+1 roots).
__global__ void oneint_kernel(int n, FuncTable ft, int natoms, const double *__restrict__ atoms, double *S, double *Tk,
                              double *V)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)n * n) return;
    const int i = (int)(t / n), j = (int)(t % n);
    const double *A = ft.origin + 3 * i, *B = ft.origin + 3 * j;
    int li[3], lj[3];
    for (int x = 0; x < 3; ++x) {
        li[x] = ft.powers[3 * i + x];
        lj[x] = ft.powers[3 * j + x];
    }
    const int Ltot = li[0] + li[1] + li[2] + lj[0] + lj[1] + lj[2];
    if (li[0] + li[1] + li[2] > 3 || lj[0] + lj[1] + lj[2] > 3) {   // f at most (the host rejects these first)
        if (S) S[t] = nan("");
        if (Tk) Tk[t] = nan("");
        if (V) V[t] = nan("");
        return;
    }
    double s_sum = 0, t_sum = 0, v_sum = 0;
    for (int p = ft.prim_off[i]; p < ft.prim_off[i + 1]; ++p)
        for (int q = ft.prim_off[j]; q < ft.prim_off[j + 1]; ++q) {
            const double a = ft.exps[p], b = ft.exps[q], g = a + b;
            double P[3], rab2 = 0;
            for (int x = 0; x < 3; ++x) {
                P[x] = (a * A[x] + b * B[x]) / g;
                rab2 += (A[x] - B[x]) * (A[x] - B[x]);
            }
            const double E = exp(-a * b / g * rab2);
            const double w = ft.cn[p] * ft.cn[q];
            // 1-D overlaps S_x[u][v], u <= li_x, v <= lj_x + 2
            double Sx[3][7][9];
            for (int x = 0; x < 3; ++x) {
                const double pa = P[x] - A[x], pb = P[x] - B[x], o2g = 0.5 / g;
                const int U = li[x], W = lj[x] + 2;
                Sx[x][0][0] = 1.0;
                for (int v = 0; v < W; ++v)
                    Sx[x][0][v + 1] = pb * Sx[x][0][v] + (v > 0 ? v * o2g * Sx[x][0][v - 1] : 0.0);
                for (int u = 0; u < U; ++u)
                    for (int v = 0; v <= W; ++v)
                        Sx[x][u + 1][v] = pa * Sx[x][u][v] + (u > 0 ? u * o2g * Sx[x][u - 1][v] : 0.0) +
                                          (v > 0 ? v * o2g * Sx[x][u][v - 1] : 0.0);
            }
            const double pre = pow(kPi / g, 1.5) * E;
            auto ov = [&](int dx, int dy, int dz) {
                return Sx[0][li[0]][lj[0] + dx] * Sx[1][li[1]][lj[1] + dy] * Sx[2][li[2]][lj[2] + dz];
            };
            const double s0 = ov(0, 0, 0);
            const int Lj = lj[0] + lj[1] + lj[2];
            double tk = b * (2 * Lj + 3) * s0 - 2.0 * b * b * (ov(2, 0, 0) + ov(0, 2, 0) + ov(0, 0, 2));
            if (lj[0] >= 2) tk -= 0.5 * lj[0] * (lj[0] - 1) * ov(-2, 0, 0);
            if (lj[1] >= 2) tk -= 0.5 * lj[1] * (lj[1] - 1) * ov(0, -2, 0);
            if (lj[2] >= 2) tk -= 0.5 * lj[2] * (lj[2] - 1) * ov(0, 0, -2);
            s_sum += w * pre * s0;
            t_sum += w * pre * tk;
            if (V) {
                const int nr = Ltot / 2 + 1;
                double vv = 0.0;
                for (int c = 0; c < natoms; ++c) {
                    const double *Cn = atoms + 4 * c;
                    double pc2 = 0;
                    for (int x = 0; x < 3; ++x) pc2 += (P[x] - Cn[x]) * (P[x] - Cn[x]);
                    const double T = g * pc2;
                    double acc = 0.0;
                    for (int r = 0; r < nr; ++r) {
                        double u, wr;
                        rys_root(nr, r, T, u, wr);
                        double prod = wr;
                        for (int x = 0; x < 3; ++x) {
                            const double c00 = (P[x] - A[x]) - u * (P[x] - Cn[x]), b10 = 0.5 * (1.0 - u) / g;
                            const int NB = li[x] + lj[x];
                            double G[8];
                            G[0] = 1.0;
                            if (NB > 0) G[1] = c00;
                            for (int k = 1; k < NB; ++k) G[k + 1] = k * b10 * G[k - 1] + c00 * G[k];
                            double sx = 0.0;
                            for (int pp = 0; pp <= lj[x]; ++pp)
                                sx += binom_d(lj[x], pp) * pow(A[x] - B[x], lj[x] - pp) * G[li[x] + pp];
                            prod *= sx;
                        }
                        acc += prod;
                    }
                    vv -= Cn[3] * acc;
                }
                v_sum += w * 2.0 * kPi / g * E * vv;
            }
        }
    const double nn = ft.norms[i] * ft.norms[j];
    if (S) S[t] = nn * s_sum;
    if (Tk) Tk[t] = nn * t_sum;
    if (V) V[t] = nn * v_sum;
}

// ---- one-electron part of the RHF nuclear gradient, one thread per (i, j):
//   2 D_ij d(T + V)_ij/dR - 2 W_ij dS_ij/dR            (PyQuante/force.py:61-64)
// Basis-centre derivatives by raising/lowering each primitive,
// d/dA_x g_a = 2 alpha g_{a+1x} - a_x g_{a-1x}; dS/dB = -dS/dA, dT/dB = -dT/dA;
// for each nucleus C the Hellmann-Feynman term dV_C/dC = -(dV_C/dA + dV_C/dB).
__device__ __forceinline__ double ov3(double (*Sx)[8][9], const int *li, const int *lj, int a0, int a1, int a2,
                                      int b0, int b1, int b2)
{
    return Sx[0][li[0] + a0][lj[0] + b0] * Sx[1][li[1] + a1][lj[1] + b1] * Sx[2][li[2] + a2][lj[2] + b2];
}

__device__ double kin3(double (*Sx)[8][9], const int *li, const int *lj, double b, int a0, int a1, int a2)
{
    const int Lj = lj[0] + lj[1] + lj[2];
    double t = b * (2 * Lj + 3) * ov3(Sx, li, lj, a0, a1, a2, 0, 0, 0) -
               2.0 * b * b * (ov3(Sx, li, lj, a0, a1, a2, 2, 0, 0) + ov3(Sx, li, lj, a0, a1, a2, 0, 2, 0) +
                              ov3(Sx, li, lj, a0, a1, a2, 0, 0, 2));
    if (lj[0] >= 2) t -= 0.5 * lj[0] * (lj[0] - 1) * ov3(Sx, li, lj, a0, a1, a2, -2, 0, 0);
    if (lj[1] >= 2) t -= 0.5 * lj[1] * (lj[1] - 1) * ov3(Sx, li, lj, a0, a1, a2, 0, -2, 0);
    if (lj[2] >= 2) t -= 0.5 * lj[2] * (lj[2] - 1) * ov3(Sx, li, lj, a0, a1, a2, 0, 0, -2);
    return t;
}

__global__ void oneint_grad_kernel(int n, FuncTable ft, int natoms, const double *__restrict__ atoms,
                                   const int *__restrict__ func_atom, const double *__restrict__ Dm,
                                   const double *__restrict__ Wm, double *grad)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (int64_t)n * n) return;
    const int i = (int)(t / n), j = (int)(t % n);
    const double *A = ft.origin + 3 * i, *B = ft.origin + 3 * j;
    int li[3], lj[3];
    for (int x = 0; x < 3; ++x) {
        li[x] = ft.powers[3 * i + x];
        lj[x] = ft.powers[3 * j + x];
    }
    if (li[0] + li[1] + li[2] > 3 || lj[0] + lj[1] + lj[2] > 3) return;   // host rejects these first
    const double nn = ft.norms[i] * ft.norms[j];
    const double d2 = 2.0 * Dm[t] * nn, w2 = 2.0 * Wm[t] * nn;
    double gA[3] = {0, 0, 0}, gB[3] = {0, 0, 0};
    const int Ltot = li[0] + li[1] + li[2] + lj[0] + lj[1] + lj[2];
    for (int p = ft.prim_off[i]; p < ft.prim_off[i + 1]; ++p)
        for (int q = ft.prim_off[j]; q < ft.prim_off[j + 1]; ++q) {
            const double a = ft.exps[p], b = ft.exps[q], g = a + b;
            double P[3], rab2 = 0;
            for (int x = 0; x < 3; ++x) {
                P[x] = (a * A[x] + b * B[x]) / g;
                rab2 += (A[x] - B[x]) * (A[x] - B[x]);
            }
            const double E = exp(-a * b / g * rab2);
            const double cw = ft.cn[p] * ft.cn[q];
            double Sx[3][8][9];
            for (int x = 0; x < 3; ++x) {
                const double pa = P[x] - A[x], pb = P[x] - B[x], o2g = 0.5 / g;
                const int U = li[x] + 1, W = lj[x] + 2;
                Sx[x][0][0] = 1.0;
                for (int v = 0; v < W; ++v) Sx[x][0][v + 1] = pb * Sx[x][0][v] + (v > 0 ? v * o2g * Sx[x][0][v - 1] : 0.0);
                for (int u = 0; u < U; ++u)
                    for (int v = 0; v <= W; ++v)
                        Sx[x][u + 1][v] = pa * Sx[x][u][v] + (u > 0 ? u * o2g * Sx[x][u - 1][v] : 0.0) +
                                          (v > 0 ? v * o2g * Sx[x][u][v - 1] : 0.0);
            }
            const double pre = cw * pow(kPi / g, 1.5) * E;
            for (int x = 0; x < 3; ++x) {
                const int dp[3] = {x == 0, x == 1, x == 2};
                double dS = 2.0 * a * ov3(Sx, li, lj, dp[0], dp[1], dp[2], 0, 0, 0);
                double dT = 2.0 * a * kin3(Sx, li, lj, b, dp[0], dp[1], dp[2]);
                if (li[x] > 0) {
                    dS -= li[x] * ov3(Sx, li, lj, -dp[0], -dp[1], -dp[2], 0, 0, 0);
                    dT -= li[x] * kin3(Sx, li, lj, b, -dp[0], -dp[1], -dp[2]);
                }
                const double c = pre * (d2 * dT - w2 * dS);
                gA[x] += c;
                gB[x] -= c;
            }
            // nuclear attraction: 1-D Rys integrals I(a', b') for a' in a-1..a+1, b' in b-1..b+1
            const int nr = (Ltot + 1) / 2 + 1;
            const double vpre = cw * 2.0 * kPi / g * E;
            for (int cnuc = 0; cnuc < natoms; ++cnuc) {
                const double *Cn = atoms + 4 * cnuc;
                double pc2 = 0;
                for (int x = 0; x < 3; ++x) pc2 += (P[x] - Cn[x]) * (P[x] - Cn[x]);
                double vA[3] = {0, 0, 0}, vB[3] = {0, 0, 0};
                for (int r = 0; r < nr; ++r) {
                    double u, wr;
                    rys_root(nr, r, g * pc2, u, wr);
                    double I0[3], IA[3], IB[3];
                    for (int x = 0; x < 3; ++x) {
                        const double c00 = (P[x] - A[x]) - u * (P[x] - Cn[x]), b10 = 0.5 * (1.0 - u) / g;
                        const int NB = li[x] + lj[x] + 2;
                        double G[10];
                        G[0] = 1.0;
                        G[1] = c00;
                        for (int k = 1; k < NB; ++k) G[k + 1] = k * b10 * G[k - 1] + c00 * G[k];
                        const double ab = A[x] - B[x];
                        // I(a', b') = sum_p C(b',p) ab^(b'-p) G[a'+p]
                        auto Iab = [&](int ap, int bp) {
                            double sx = 0.0;
                            for (int pp = 0; pp <= bp; ++pp) sx += binom_d(bp, pp) * pow(ab, bp - pp) * G[ap + pp];
                            return sx;
                        };
                        I0[x] = Iab(li[x], lj[x]);
                        IA[x] = 2.0 * a * Iab(li[x] + 1, lj[x]) - (li[x] > 0 ? li[x] * Iab(li[x] - 1, lj[x]) : 0.0);
                        IB[x] = 2.0 * b * Iab(li[x], lj[x] + 1) - (lj[x] > 0 ? lj[x] * Iab(li[x], lj[x] - 1) : 0.0);
                    }
                    vA[0] += wr * IA[0] * I0[1] * I0[2];
                    vA[1] += wr * I0[0] * IA[1] * I0[2];
                    vA[2] += wr * I0[0] * I0[1] * IA[2];
                    vB[0] += wr * IB[0] * I0[1] * I0[2];
                    vB[1] += wr * I0[0] * IB[1] * I0[2];
                    vB[2] += wr * I0[0] * I0[1] * IB[2];
                }
                const double zf = -Cn[3] * vpre * d2;   // V_C = -Z_C <..>, times 2 D_ij
                for (int x = 0; x < 3; ++x) {
                    gA[x] += zf * vA[x];
                    gB[x] += zf * vB[x];
                    atomicAdd(grad + 3 * cnuc + x, -zf * (vA[x] + vB[x]));
                }
            }
        }
    const int ai = func_atom[i], aj = func_atom[j];
    for (int x = 0; x < 3; ++x) {
        atomicAdd(grad + 3 * ai + x, gA[x]);
        atomicAdd(grad + 3 * aj + x, gB[x]);
    }
}

// ---- allocation-free one-electron integrals (pqb_oneint_noalloc) --------
// Scratch for the packed atom table {x, y, z, Z} that oneint_kernel reads:
// a file-scope device array, so the entry point needs no cudaMalloc.  Every
// GPU that loads this library holds it (128 KiB) until the process exits.
#define PQB_NOALLOC_MAX_ATOMS 4096
#define PQB_NOALLOC_MAX_DEVICES 64
static __device__ __align__(256) double pqb_noalloc_atoms[4 * PQB_NOALLOC_MAX_ATOMS];

__global__ void pack_atoms_kernel(int natoms, const double *__restrict__ xyz, const double *__restrict__ z,
                                  double *out)
{
    int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= natoms) return;
    out[4 * a + 0] = xyz[3 * a + 0];
    out[4 * a + 1] = xyz[3 * a + 1];
    out[4 * a + 2] = xyz[3 * a + 2];
    out[4 * a + 3] = z[a];
}

// ---- stored-integral J/K: one block per packed bra row IJ (i >= j); the row
// holds (ij|kl) for every kl <= ij, contiguous.  Same unique-quartet
// digestion as EpiJK.
__global__ void jk_packed_kernel(const double *__restrict__ ints, const double *__restrict__ D, double *Jacc,
                                 double *Kacc, int n)
{
    const int64_t IJ = blockIdx.x;
    int i = (int)((sqrt(8.0 * (double)IJ + 1.0) - 1.0) * 0.5);
    while ((int64_t)i * (i + 1) / 2 > IJ) --i;
    while ((int64_t)(i + 1) * (i + 2) / 2 <= IJ) ++i;
    const int j = (int)(IJ - (int64_t)i * (i + 1) / 2);
    const double *row = ints + IJ * (IJ + 1) / 2;
    const double Dij = D[(int64_t)i * n + j];
    double jij = 0.0;
    for (int64_t KL = threadIdx.x; KL <= IJ; KL += blockDim.x) {
        int k = (int)((sqrt(8.0 * (double)KL + 1.0) - 1.0) * 0.5);
        while ((int64_t)k * (k + 1) / 2 > KL) --k;
        while ((int64_t)(k + 1) * (k + 2) / 2 <= KL) ++k;
        const int l = (int)(KL - (int64_t)k * (k + 1) / 2);
        const double v = row[KL] * (i == j ? 0.5 : 1.0) * (k == l ? 0.5 : 1.0) * (IJ == KL ? 0.5 : 1.0);
        jij += v * D[(int64_t)k * n + l];
        atomicAdd(Jacc + (int64_t)k * n + l, 2.0 * v * Dij);
        atomicAdd(Kacc + (int64_t)i * n + k, v * D[(int64_t)j * n + l]);
        atomicAdd(Kacc + (int64_t)i * n + l, v * D[(int64_t)j * n + k]);
        atomicAdd(Kacc + (int64_t)j * n + k, v * D[(int64_t)i * n + l]);
        atomicAdd(Kacc + (int64_t)j * n + l, v * D[(int64_t)i * n + k]);
    }
    __shared__ double red[32];
    for (int o = 16; o > 0; o >>= 1) jij += __shfl_down_sync(0xffffffffu, jij, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = jij;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
        atomicAdd(Jacc + (int64_t)i * n + j, 2.0 * s);
    }
}

// ---- stored-integral J/K, register form (the HBM-bound path for
// nbf <= 32 * MAXM).  A CTA owns the packed rows IJ = (i, j), j in
// [j0, j0 + 16), of one i; warp w owns rows j0 + w and j0 + w + 8.  The
// warps walk the columns KL = (k, l) segment by segment (k fixed, lane
// owns l = lane + 32 m), reading every integral once with coalesced loads.
// With v' the degeneracy-weighted integral:
//   Jacc[i,j] += 2 v' D_kl   per-row register sums
//   Jacc[k,l] += 2 v' D_ij   per-warp partials in shared memory, summed
//                            over the CTA's rows once per segment
//   Kacc[i,l] += v' D_jk     register row accI[m] (lane-owned columns)
//   Kacc[i,k] += v' D_jl     per-segment partials over 8 lane groups, parked
//                            in a shared ring and folded into column k of
//                            accI once per 32-segment block
//   Kacc[j,l] += v' D_ik     register rows accJ[q][m]
//   Kacc[j,k] += v' D_il     the same, into column k of accJ
// The register rows go to Kacc once per CTA (accI summed over the warps).
constexpr int kRgWarps = 8, kRgRPW = 2, kRgRows = kRgWarps * kRgRPW, kRgPrefetch = 3;
// segment-sum ring: kRgNv values (row i, rows j_q) x kRgParts partials x 32
// columns, rows padded to 33 so that the writers hit distinct banks
constexpr int kRgParts = 8;
constexpr int kRgNv = 1 + kRgRPW, kRgRingPitch = 33, kRgRing = kRgNv * kRgParts * kRgRingPitch;

__device__ __forceinline__ double warp_sum(double x)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// L2 prefetch of the 16-byte aligned interior of [p, p + len) (a hint: no
// data returns to the SM; the range lies inside the packed array).
__device__ __forceinline__ void prefetch_l2(const double *p, int len)
{
    const uintptr_t a = ((uintptr_t)p + 15) & ~(uintptr_t)15, b = ((uintptr_t)(p + len)) & ~(uintptr_t)15;
    if (b > a)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(__cvta_generic_to_global((const void *)a)),
                     "r"((unsigned)(b - a))
                     : "memory");
}

// Per-warp state of a tile: the warp's rows j (q = 0 .. kRgRPW-1), the row
// weights wq (1/2 on the diagonal row j = i, 0 past i) and the register rows.
// The weights wq are applied to the row constants and, for accJ and jrow,
// once at the end, so the per-integral loop multiplies only the column
// weights (1/2 at l = k, and at kl = ij in the last segment).
template <int MAXM> struct RgRows {
    const double *rowp[kRgRPW], *Djp[kRgRPW];
    int jq[kRgRPW];
    bool okq[kRgRPW];
    double Dij2[kRgRPW], wq[kRgRPW], jrow[kRgRPW], accJ[kRgRPW][MAXM], accI[MAXM];
};

template <int... Is, class F>
__device__ __forceinline__ void rg_static_for(std::integer_sequence<int, Is...>, F &&f)
{
    (f(std::integral_constant<int, Is>{}), ...);
}

// Jacc[k, l] for l <= k from the CTA's per-warp column partials of one
// segment (one barrier per segment; the partials are double-buffered).
__device__ __forceinline__ void rg_column_sums(const double *jcb, int stride, double *Jacc, int n, int k)
{
    __syncthreads();
    for (int l = threadIdx.x; l <= k; l += kRgWarps * 32) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < kRgWarps; ++w) s += jcb[w * stride + l];
        if (s != 0.0) atomicAdd(Jacc + (int64_t)k * n + l, s);
    }
}

// Segment k (< i) of the warp's rows, k in [32 KB, 32 KB + 31]: the chunk
// count KB + 1 and the register slot KB of column k are compile-time, so the
// register rows stay in registers and the segment sums are plain adds.
template <int MAXM, int KB>
__device__ __forceinline__ void rg_segment(RgRows<MAXM> &r, const double *__restrict__ D, const double *Di,
                                           double *jcw, double *ring, int n, int i, int k, int lane)
{
    const int KL0 = k * (k + 1) / 2;
    const double *Dk = D + (int64_t)k * n;
    const double Dik = __ldg(Di + k);
    double Djk[kRgRPW], kik[kRgRPW], kjk[kRgRPW];
#pragma unroll
    for (int q = 0; q < kRgRPW; ++q) {
        Djk[q] = r.wq[q] * __ldg(r.Djp[q] + k);
        kik[q] = 0.0;
        kjk[q] = 0.0;
    }
#pragma unroll
    for (int m = 0; m <= KB; ++m) {
        const int l = 32 * m + lane;
        const bool inseg = m < KB || l <= k;
        const double Dkl = inseg ? __ldg(Dk + l) : 0.0;
        const double Dil = inseg ? __ldg(Di + l) : 0.0;
        double jcol = 0.0;
#pragma unroll
        for (int q = 0; q < kRgRPW; ++q) {
            const bool ok = r.okq[q] && inseg;
            double v = ok ? __ldg(r.rowp[q] + KL0 + l) : 0.0;
            const double Djl = ok ? __ldg(r.Djp[q] + l) : 0.0;
            if (m == KB && l == k) v *= 0.5;
            r.jrow[q] = fma(v, Dkl, r.jrow[q]);
            jcol = fma(v, r.Dij2[q], jcol);
            kik[q] = fma(v, Djl, kik[q]);
            r.accI[m] = fma(v, Djk[q], r.accI[m]);
            kjk[q] = fma(v, Dil, kjk[q]);
            r.accJ[q][m] = fma(v, Dik, r.accJ[q][m]);
        }
        jcw[l] = jcol;
    }
    // the segment sums Kacc[i,k] (value 0) and Kacc[j_q,k] (value 1 + q):
    // butterfly levels down to kRgParts leave lane p < kRgParts with the sum
    // over lanes p + kRgParts t, parked in the warp's ring until the
    // 32-segment block is folded
    double sv[kRgNv];
    sv[0] = 0.0;
#pragma unroll
    for (int q = 0; q < kRgRPW; ++q) {
        sv[0] = fma(r.wq[q], kik[q], sv[0]);
        sv[1 + q] = kjk[q];
    }
#pragma unroll
    for (int v = 0; v < kRgNv; ++v)
#pragma unroll
        for (int o = 16; o >= kRgParts; o >>= 1) sv[v] += __shfl_xor_sync(0xffffffffu, sv[v], o);
    if (lane < kRgParts) {
#pragma unroll
        for (int v = 0; v < kRgNv; ++v) ring[(v * kRgParts + lane) * kRgRingPitch + (k & 31)] = sv[v];
    }
}

// Fold a finished 32-segment block KB out of the ring: lane c adds the kRgParts
// partials of column 32 KB + c to its register slot KB (compile-time).
template <int MAXM, int KB>
__device__ __forceinline__ void rg_fold_block(RgRows<MAXM> &r, const double *ring, int kend, int lane)
{
    __syncwarp();
    if (32 * KB + lane <= kend) {
        double s[kRgNv];
#pragma unroll
        for (int v = 0; v < kRgNv; ++v) {
            s[v] = 0.0;
#pragma unroll
            for (int p = 0; p < kRgParts; ++p) s[v] += ring[(v * kRgParts + p) * kRgRingPitch + lane];
        }
        r.accI[KB] += s[0];
#pragma unroll
        for (int q = 0; q < kRgRPW; ++q) r.accJ[q][KB] += s[1 + q];
    }
    __syncwarp();
}

// The last segment k = i: row (i, j) holds kl <= (i, j), so only l <= j,
// with weight 1/2 at kl = ij.  Runs once per tile; the slot of column k is
// a run-time index here.
template <int MAXM>
__device__ __forceinline__ void rg_last_segment(RgRows<MAXM> &r, const double *__restrict__ D, const double *Di,
                                                double *jcw, int n, int i, int lane)
{
    const int k = i, KL0 = k * (k + 1) / 2;
    const double *Dk = D + (int64_t)k * n;
    const double Dik = __ldg(Di + k);
    double Djk[kRgRPW], kik[kRgRPW], kjk[kRgRPW];
    int lmax[kRgRPW];
#pragma unroll
    for (int q = 0; q < kRgRPW; ++q) {
        Djk[q] = r.wq[q] * __ldg(r.Djp[q] + k);
        kik[q] = 0.0;
        kjk[q] = 0.0;
        lmax[q] = r.okq[q] ? r.jq[q] : -1;   // rows past i load nothing
    }
#pragma unroll
    for (int m = 0; m < MAXM; ++m) {
        if (32 * m > k) continue;   // warp-uniform: chunks past the segment are skipped
        const int l = 32 * m + lane;
        const bool inseg = l <= k;
        const double Dkl = inseg ? __ldg(Dk + l) : 0.0;
        const double Dil = inseg ? __ldg(Di + l) : 0.0;
        const double wkl = l == k ? 0.5 : 1.0;
        double jcol = 0.0;
#pragma unroll
        for (int q = 0; q < kRgRPW; ++q) {
            const bool ok = l <= lmax[q];
            double v = ok ? __ldg(r.rowp[q] + KL0 + l) : 0.0;
            const double Djl = ok ? __ldg(r.Djp[q] + l) : 0.0;
            v *= wkl * (l == r.jq[q] ? 0.5 : 1.0);
            r.jrow[q] = fma(v, Dkl, r.jrow[q]);
            jcol = fma(v, r.Dij2[q], jcol);
            kik[q] = fma(v, Djl, kik[q]);
            r.accI[m] = fma(v, Djk[q], r.accI[m]);
            kjk[q] = fma(v, Dil, kjk[q]);
            r.accJ[q][m] = fma(v, Dik, r.accJ[q][m]);
        }
        jcw[l] = jcol;
    }
    double ki = 0.0;
#pragma unroll
    for (int q = 0; q < kRgRPW; ++q) ki = fma(r.wq[q], kik[q], ki);
    const double sk = warp_sum(ki);
    double sj[kRgRPW];
#pragma unroll
    for (int q = 0; q < kRgRPW; ++q) sj[q] = warp_sum(kjk[q]);
    // (as multiply-adds by a 0/1 factor: a conditional add with a run-time
    // slot would let the compiler turn the unrolled rows into an indexed,
    // memory-resident array)
    const int kslot = lane == (k & 31) ? (k >> 5) : -1;
#pragma unroll
    for (int m = 0; m < MAXM; ++m) {
        const double f = m == kslot ? 1.0 : 0.0;
        r.accI[m] = fma(f, sk, r.accI[m]);
#pragma unroll
        for (int q = 0; q < kRgRPW; ++q) r.accJ[q][m] = fma(f, sj[q], r.accJ[q][m]);
    }
}

template <int MAXM>
__global__ void __launch_bounds__(kRgWarps * 32) jk_packed_reg_kernel(const double *__restrict__ ints,
                                                                      const double *__restrict__ D, double *Jacc,
                                                                      double *Kacc, int n,
                                                                      const int2 *__restrict__ tiles, int ntiles)
{
    // column partials of a segment, double-buffered: jc[2][kRgWarps][MAXM * 32];
    // per-warp rows i, summed at the end: kis[kRgWarps][MAXM * 32]
    extern __shared__ double rg_smem[];
    constexpr int kStride = MAXM * 32;
    double *jc = rg_smem;
    double(*kis)[kStride] = reinterpret_cast<double(*)[kStride]>(rg_smem + 2 * kRgWarps * kStride);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // per-warp ring of segment-sum partials: [value][partial p][column k % 32]
    double *ring = rg_smem + 3 * kRgWarps * kStride + warp * kRgRing;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int i = tiles[t].x, j0 = tiles[t].y;
        const int64_t I0 = (int64_t)i * (i + 1) / 2;
        const double *Di = D + (int64_t)i * n;
        RgRows<MAXM> r;
#pragma unroll
        for (int q = 0; q < kRgRPW; ++q) {
            const int j = j0 + warp + kRgWarps * q;
            r.okq[q] = j <= i;
            r.jq[q] = r.okq[q] ? j : i;
            const int64_t IJ = I0 + r.jq[q];
            r.rowp[q] = ints + IJ * (IJ + 1) / 2;
            r.Djp[q] = D + (int64_t)r.jq[q] * n;
            r.wq[q] = r.okq[q] ? (i == r.jq[q] ? 0.5 : 1.0) : 0.0;   // rows past i contribute nothing
            r.Dij2[q] = 2.0 * r.wq[q] * __ldg(Di + r.jq[q]);
            r.jrow[q] = 0.0;
#pragma unroll
            for (int m = 0; m < MAXM; ++m) r.accJ[q][m] = 0.0;
        }
#pragma unroll
        for (int m = 0; m < MAXM; ++m) r.accI[m] = 0.0;
        // lane q < kRgRPW prefetches row q: segment kk of it into L2
        const double *pf_row = r.rowp[0];
        bool pf_ok = r.okq[0];
        int pf_j = r.jq[0];
#pragma unroll
        for (int q = 1; q < kRgRPW; ++q)
            if (lane == q) pf_row = r.rowp[q], pf_ok = r.okq[q], pf_j = r.jq[q];
        pf_ok = pf_ok && lane < kRgRPW;
        if (pf_ok)
            for (int kk = 0; kk < kRgPrefetch && kk <= i; ++kk)
                prefetch_l2(pf_row + kk * (kk + 1) / 2, kk < i ? kk + 1 : pf_j + 1);
        int buf = 0;
        rg_static_for(std::make_integer_sequence<int, MAXM>{}, [&](auto kbc) {
            constexpr int KB = decltype(kbc)::value;
            if (32 * KB >= i) return;
            const int kend = min(32 * KB + 31, i - 1);
            for (int k = 32 * KB; k <= kend; ++k) {
                if (pf_ok && k + kRgPrefetch <= i) {
                    const int kk = k + kRgPrefetch;
                    prefetch_l2(pf_row + kk * (kk + 1) / 2, kk < i ? kk + 1 : pf_j + 1);
                }
                double *jcb = jc + buf * kRgWarps * kStride;
                rg_segment<MAXM, KB>(r, D, Di, jcb + warp * kStride, ring, n, i, k, lane);
                rg_column_sums(jcb, kStride, Jacc, n, k);
                buf ^= 1;
            }
            rg_fold_block<MAXM, KB>(r, ring, kend, lane);
        });
        {
            double *jcb = jc + buf * kRgWarps * kStride;
            rg_last_segment<MAXM>(r, D, Di, jcb + warp * kStride, n, i, lane);
            rg_column_sums(jcb, kStride, Jacc, n, i);
        }
#pragma unroll
        for (int q = 0; q < kRgRPW; ++q) {
            const double x = warp_sum(r.jrow[q]);
            if (lane == 0 && r.okq[q] && x != 0.0) atomicAdd(Jacc + (int64_t)i * n + r.jq[q], 2.0 * r.wq[q] * x);
        }
        // rows j of Kacc from registers; row i summed over the warps
#pragma unroll
        for (int m = 0; m < MAXM; ++m) {
            const int c = 32 * m + lane;
            kis[warp][c] = r.accI[m];
            if (c <= i) {
#pragma unroll
                for (int q = 0; q < kRgRPW; ++q)
                    if (r.okq[q] && r.accJ[q][m] != 0.0)
                        atomicAdd(Kacc + (int64_t)r.jq[q] * n + c, r.wq[q] * r.accJ[q][m]);
            }
        }
        __syncthreads();
        for (int c = threadIdx.x; c <= i; c += kRgWarps * 32) {
            double s = 0.0;
#pragma unroll
            for (int w = 0; w < kRgWarps; ++w) s += kis[w][c];
            if (s != 0.0) atomicAdd(Kacc + (int64_t)i * n + c, s);
        }
        __syncthreads();
    }
}

template <int MAXM>
static cudaError_t launch_packed_reg(const double *ints, const double *D, double *J, double *K, int nbf,
                                     const int2 *tiles, int ntiles, int grid, cudaStream_t st)
{
    const size_t smem = sizeof(double) * (3 * kRgWarps * MAXM * 32 + kRgWarps * kRgRing);
    cudaError_t e = cudaFuncSetAttribute(jk_packed_reg_kernel<MAXM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return e;
    jk_packed_reg_kernel<MAXM><<<grid, kRgWarps * 32, smem, st>>>(ints, D, J, K, nbf, tiles, ntiles);
    return cudaGetLastError();
}

__global__ void boys_eval_kernel(int m, int count, const double *T, double *F)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    double f[17];
    boys_rt(m, T[t], f);
    for (int k = 0; k <= m; ++k) F[(int64_t)t * (m + 1) + k] = f[k];
}

// F_0 .. F_lt by the branch-free compact-row form of the thread-mode kernels
// (boys_os)
__global__ void boys_rows_eval_kernel(int lt, int count, const double *T, double *F)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    double f[5];
    switch (lt) {
    case 0: boys_os<0>(T[t], f); break;
    case 1: boys_os<1>(T[t], f); break;
    case 2: boys_os<2>(T[t], f); break;
    case 3: boys_os<3>(T[t], f); break;
    default: boys_os<4>(T[t], f); break;
    }
    for (int k = 0; k <= lt; ++k) F[(int64_t)t * (lt + 1) + k] = f[k];
}

__global__ void rys_eval_kernel(int nr, int count, const double *T, double *u, double *w)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    double uu[5], ww[5];
    // the same evaluation the Fock-build kernels use (moments for 1-2 roots, tables above)
    switch (nr) {
    case 1: rys_roots_fast<1>(T[t], uu, ww); break;
    case 2: rys_roots_fast<2>(T[t], uu, ww); break;
    case 3: rys_roots_fast<3>(T[t], uu, ww); break;
    case 4: rys_roots_fast<4>(T[t], uu, ww); break;
    default: rys_roots_fast<5>(T[t], uu, ww); break;
    }
    for (int r = 0; r < nr; ++r) {
        u[(int64_t)t * nr + r] = uu[r];
        w[(int64_t)t * nr + r] = ww[r];
    }
}

// FP64 FMA probe: 8 independent chains per thread keep the DFMA pipe full.
__global__ void dfma_probe_kernel(int iters, double *sink)
{
    double a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = threadIdx.x * 1e-3 + k;
    const double b = 0.999999, c = 1e-9;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) a[k] = fma(a[k], b, c);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += a[k];
    if (s == 12345.678) sink[0] = s;   // never true; keeps the chains live
}

__global__ void finalize_q_kernel(const unsigned long long *q2, double *Q, int np)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < np) Q[t] = sqrt(__longlong_as_double((long long)q2[t]));
}

// ====================================================================== host

static inline int64_t pair_idx64(int64_t i, int64_t j) { return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i; }

// Run f(0) .. f(n - 1) on up to nthreads threads (tasks handed out in
// order).  Returns false if a task threw (a host allocation failure): no
// exception crosses the C ABI, and the remaining tasks are not started.
template <class F> static bool run_tasks(int n, int nthreads, F f)
{
    nthreads = std::max(1, std::min(nthreads, n));
    std::atomic<bool> failed{false};
    std::atomic<int> next{0};
    auto worker = [&] {
        for (int i = next++; i < n && !failed.load(); i = next++) {
            try {
                f(i);
            } catch (...) {
                failed.store(true);
            }
        }
    };
    if (nthreads == 1) {
        worker();
        return !failed.load();
    }
    std::vector<std::thread> pool;
    try {
        for (int t = 0; t < nthreads; ++t) pool.emplace_back(worker);
    } catch (...) {
        failed.store(true);   // no thread could be started: the running ones stop early
    }
    for (auto &th : pool) th.join();
    return !failed.load();
}

static int host_threads()
{
    const unsigned hw = std::thread::hardware_concurrency();
    return (int)std::min(32u, std::max(1u, hw));
}

extern "C" {

int pqb_version(void) { return 1; }

int64_t pqb_ijkl2intindex(int64_t i, int64_t j, int64_t k, int64_t l)
{
    int64_t ij = pair_idx64(i, j), kl = pair_idx64(k, l);
    return ij >= kl ? ij * (ij + 1) / 2 + kl : kl * (kl + 1) / 2 + ij;
}

int pqb_create(pqb_ctx **out, int device)
{
    if (!out) return PQB_E_ARG;
    *out = nullptr;
    pqb_ctx *ctx = new (std::nothrow) pqb_ctx();
    if (!ctx) return PQB_E_NOMEM;
    ctx->device = device;
    for (int c = 0; c < kNumQuartetClass; ++c) ctx->chunk[c] = kDefaultChunk;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
        delete ctx;
        return PQB_E_CUDA;
    }
    cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, device);
    *out = ctx;
    return PQB_OK;
}

static cudaError_t ensure_streams(pqb_ctx *ctx)
{
    if (ctx->ev_fork) return cudaSuccess;
    for (int k = 0; k < pqb_ctx::kStreams; ++k) {
        cudaError_t e = cudaStreamCreateWithFlags(&ctx->streams[k], cudaStreamNonBlocking);
        if (e != cudaSuccess) return e;
        e = cudaEventCreateWithFlags(&ctx->ev_join[k], cudaEventDisableTiming);
        if (e != cudaSuccess) return e;
    }
    return cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming);
}

static void drop_graphs(pqb_ctx *ctx)
{
    for (int gi = 0; gi < 6; ++gi) {
        if (ctx->graph_exec[gi]) cudaGraphExecDestroy(ctx->graph_exec[gi]);
        ctx->graph_exec[gi] = nullptr;
        ctx->graph_warm[gi] = false;
    }
}

static void release_basis(pqb_ctx *ctx)
{
    drop_graphs(ctx);
    free_dev(ctx->d_Jacc);
    free_dev(ctx->d_Kacc);
    free_dev(ctx->d_Jacc2);
    free_dev(ctx->d_Kacc2);
    ctx->d_Jacc = ctx->d_Kacc = ctx->d_Jacc2 = ctx->d_Kacc2 = nullptr;
    free_dev(ctx->d_hD);
    free_dev(ctx->d_hG);
    free_dev(ctx->d_hJ);
    free_dev(ctx->d_hK);
    ctx->d_hD = ctx->d_hG = ctx->d_hJ = ctx->d_hK = nullptr;
    free_dev(ctx->d_Dscaled2);
    free_dev(ctx->d_Dscaled2_f);
    ctx->d_Dscaled2 = nullptr;
    ctx->d_Dscaled2_f = nullptr;
    free_dev(ctx->d_pairs);
    free_dev(ctx->d_prims);
    free_dev(ctx->d_fscale);
    free_dev(ctx->d_escale);
    free_dev(ctx->d_Dscaled);
    free_dev(ctx->d_Dscaled_f);
    ctx->d_escale = nullptr;
    ctx->d_Dscaled = nullptr;
    ctx->d_Dscaled_f = nullptr;
    free_dev(ctx->d_q2);
    free_dev(ctx->d_Qpair);
    free_dev(ctx->d_shell_info);
    ctx->d_Qpair = nullptr;
    ctx->d_shell_info = nullptr;
    ctx->scr.dmax = nullptr;   // the bounds are per shell of the old basis
    ctx->scr.Qpair = nullptr;
    free_dev(ctx->d_full);
    free_dev(ctx->d_diag);
    free_dev(ctx->d_plan);
    free_dev(ctx->d_shell_atom);
    free_dev(ctx->d_mol_off);
    free_dev(ctx->d_mol_n);
    ctx->d_shell_atom = nullptr;
    ctx->d_mol_off = nullptr;
    ctx->d_mol_n = nullptr;
    ctx->d_pairs = nullptr;
    ctx->d_prims = nullptr;
    ctx->d_fscale = nullptr;
    ctx->d_q2 = nullptr;
    ctx->d_full = ctx->d_diag = ctx->d_plan = nullptr;
    ctx->plan_cap = 0;
    ctx->have_q = ctx->have_plan = false;
}

void pqb_destroy(pqb_ctx *ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    release_basis(ctx);
    free_dev(ctx->d_atoms);
    free_dev(ctx->d_pk_tiles);
    for (int k = 0; k < pqb_ctx::kStreams; ++k) {
        if (ctx->streams[k]) cudaStreamDestroy(ctx->streams[k]);
        if (ctx->ev_join[k]) cudaEventDestroy(ctx->ev_join[k]);
    }
    if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
    if (ctx->cap_stream) cudaStreamDestroy(ctx->cap_stream);
    delete ctx;
}

int pqb_last_error(const pqb_ctx *ctx, char *buf, size_t len)
{
    if (!ctx || !buf || len == 0) return PQB_E_ARG;
    snprintf(buf, len, "%s", ctx->err.c_str());
    return PQB_OK;
}

int pqb_num_pairs(const pqb_ctx *ctx) { return ctx ? (int)ctx->pairs.size() : 0; }

// Bucket work items by class.  Within a class the items go by descending
// primitive-quartet count (block-mode kernels advance their items in lockstep
// over primitive quartets; thread-mode warps get similar trip counts), then by
// bra pair, then in generation order (ket pair ascending), so neighbouring
// lanes share the bra and often the ket's first shell and the J/K epilogue's
// warp runs are long.  Two stable counting sorts (bra pair, then count) keep
// this linear in the number of items, which reaches 5e8 for batched bases.
// The items of one class, given as segments in generation order, into dst
// ordered by descending count, then bra pair, then generation order.
static void order_class_items(const std::vector<const std::vector<int4> *> &segs, int4 *dst)
{
    size_t n = 0;
    int maxp = 1, maxbra = 0;
    for (auto *v : segs) {
        n += v->size();
        for (auto &e : *v) {
            maxp = std::max(maxp, e.w);
            maxbra = std::max(maxbra, e.x);
        }
    }
    if (n == 0) return;
    std::vector<int4> bybra(n);
    {
        std::vector<int64_t> hist((size_t)maxbra + 2, 0);
        for (auto *v : segs)
            for (auto &e : *v) hist[e.x + 1]++;
        for (size_t k = 1; k < hist.size(); ++k) hist[k] += hist[k - 1];
        for (auto *v : segs)
            for (auto &e : *v) bybra[hist[e.x]++] = e;
    }
    std::vector<int64_t> hist(maxp + 2, 0);
    for (auto &e : bybra) hist[maxp - e.w]++;
    int64_t s = 0;
    for (auto &h : hist) {
        int64_t t = h;
        h = s;
        s += t;
    }
    for (auto &e : bybra) dst[hist[maxp - e.w]++] = e;
}

static void bucket_sorted(std::vector<std::vector<int4>> &cls, std::vector<int4> &flat, int64_t *off, int64_t *cnt)
{
    flat.clear();
    for (int c = 0; c < kNumQuartetClass; ++c) {
        off[c] = (int64_t)flat.size();
        cnt[c] = (int64_t)cls[c].size();
        flat.resize(flat.size() + cls[c].size());
        order_class_items({&cls[c]}, flat.data() + off[c]);
    }
}

static inline int4 oriented_quartet(const std::vector<PairInfo> &pairs, int p, int q, int &qc)
{
    int cp = pairs[p].cls, cq = pairs[q].cls;
    if (cp < cq) {
        std::swap(p, q);
        std::swap(cp, cq);
    }
    qc = quartet_class(cp, cq);
    return make_int4(p, q, 0, pairs[p].nprim * pairs[q].nprim);
}

int pqb_shells_upload(pqb_ctx *ctx, int nshell, const int *shell_l, const int *shell_nprim, const int *prim_off,
                      const int *shell_f0, const double *shell_xyz, const double *prim_exp, const double *prim_coef,
                      int nbf, const double *fscale)
{
    const int mol_shell_off[2] = {0, nshell};
    return pqb_shells_upload_batch(ctx, 1, mol_shell_off, nshell, shell_l, shell_nprim, prim_off, shell_f0, shell_xyz,
                                   prim_exp, prim_coef, nbf, fscale);
}

static int shells_upload_batch_impl(pqb_ctx *ctx, int nmol, const int *mol_shell_off, int nshell, const int *shell_l,
                                    const int *shell_nprim, const int *prim_off, const int *shell_f0, const double *shell_xyz,
                                    const double *prim_exp, const double *prim_coef, int nbf, const double *fscale)
{
    if (!ctx || nmol <= 0 || !mol_shell_off || nshell <= 0 || !shell_l || !shell_nprim || !prim_off || !shell_f0 ||
        !shell_xyz || !prim_exp || !prim_coef || !fscale || nbf <= 0)
        return fail(ctx, PQB_E_ARG, "pqb_shells_upload: bad arguments");
    if (mol_shell_off[0] != 0 || mol_shell_off[nmol] != nshell)
        return fail(ctx, PQB_E_SHAPE, "molecule shell offsets must run from 0 to nshell");
    for (int m = 0; m < nmol; ++m)
        if (mol_shell_off[m + 1] <= mol_shell_off[m]) return fail(ctx, PQB_E_SHAPE, "molecule %d has no shells", m);
    PQB_CK(ctx, cudaSetDevice(ctx->device));
    release_basis(ctx);
    int nf = 0;
    for (int s = 0; s < nshell; ++s) {
        if (shell_l[s] < 0 || shell_l[s] > kMaxL)
            return fail(ctx, PQB_E_CLASS, "shell %d: angular momentum %d > %d (s, p, d supported)", s, shell_l[s],
                        kMaxL);
        if (shell_nprim[s] <= 0 || shell_nprim[s] > 64)
            return fail(ctx, PQB_E_NPRIM, "shell %d: %d primitives (1..64 supported)", s, shell_nprim[s]);
        if (shell_f0[s] != nf) return fail(ctx, PQB_E_SHAPE, "shell %d: functions not consecutive", s);
        nf += ncart(shell_l[s]);
    }
    if (nf != nbf) return fail(ctx, PQB_E_SHAPE, "shells cover %d functions, nbf = %d", nf, nbf);
    ctx->nbf = nbf;
    ctx->nshell = nshell;
    ctx->nmol = nmol;
    ctx->mol_f0.assign(nmol, 0);
    ctx->mol_n.assign(nmol, 0);
    ctx->mol_off.assign(nmol, 0);
    long long off = 0;
    std::vector<int> shell_mol(nshell);
    for (int m = 0; m < nmol; ++m) {
        const int s0 = mol_shell_off[m], s1 = mol_shell_off[m + 1];
        ctx->mol_f0[m] = shell_f0[s0];
        ctx->mol_n[m] = shell_f0[s1 - 1] + ncart(shell_l[s1 - 1]) - shell_f0[s0];
        ctx->mol_off[m] = off;
        off += (long long)ctx->mol_n[m] * ctx->mol_n[m];
        for (int sh = s0; sh < s1; ++sh) shell_mol[sh] = m;
    }
    ctx->dense_len = off;
    // pairs
    std::vector<PairInfo> pairs;
    std::vector<PrimPair> prims;
    pairs.reserve((size_t)nshell * (nshell + 1) / 2);
    ctx->pair_first.clear();
    for (int a = 0; a < nshell; ++a)
        for (int b = mol_shell_off[shell_mol[a]]; b <= a; ++b) {
            int s1 = a, s2 = b;
            if (shell_l[s2] > shell_l[s1]) std::swap(s1, s2);
            PairInfo pi{};
            const double *A = shell_xyz + 3 * s1, *B = shell_xyz + 3 * s2;
            double r2 = 0;
            for (int x = 0; x < 3; ++x) {
                pi.A[x] = A[x];
                pi.AB[x] = A[x] - B[x];
                r2 += pi.AB[x] * pi.AB[x];
            }
            pi.prim_off = (int)prims.size();
            for (int p = prim_off[s1]; p < prim_off[s1] + shell_nprim[s1]; ++p)
                for (int q = prim_off[s2]; q < prim_off[s2] + shell_nprim[s2]; ++q) {
                    const double al = prim_exp[p], be = prim_exp[q], z = al + be;
                    const double e = exp(-al * be / z * r2);
                    // keep unless the pair's overlap weight is below 1e-20
                    if (fabs(prim_coef[p] * prim_coef[q]) * e * pow(kPi / z, 1.5) < 1e-20) continue;
                    PrimPair pp{};
                    pp.zeta = z;
                    pp.izeta = 1.0 / z;
                    for (int x = 0; x < 3; ++x) pp.P[x] = (al * A[x] + be * B[x]) / z;
                    pp.K = prim_coef[p] * prim_coef[q] * kPairPre / z * e;
                    pp.alpha_a = al;
                    pp.f[0] = (float)pp.zeta;
                    pp.f[1] = (float)pp.izeta;
                    for (int x = 0; x < 3; ++x) pp.f[2 + x] = (float)pp.P[x];
                    pp.f[5] = (float)pp.K;
                    prims.push_back(pp);
                }
            pi.nprim = (int)prims.size() - pi.prim_off;
            pi.fa = shell_f0[s1];
            pi.fb = shell_f0[s2];
            pi.sa = s1;
            pi.sb = s2;
            pi.la = shell_l[s1];
            pi.lb = shell_l[s2];
            pi.cls = pair_class(pi.la, pi.lb);
            const int m = shell_mol[a];
            pi.nm = ctx->mol_n[m];
            pi.mol = m;
            pi.bo = ctx->mol_off[m] - (long long)ctx->mol_f0[m] * (ctx->mol_n[m] + 1);
            pairs.push_back(pi);
        }
    // first pair of each molecule (pairs are generated molecule by molecule)
    {
        std::vector<int> first_of_mol(nmol, -1);
        ctx->pair_first.resize(pairs.size());
        for (size_t p = 0; p < pairs.size(); ++p) {
            const int m = shell_mol[pairs[p].sa];
            if (first_of_mol[m] < 0) first_of_mol[m] = (int)p;
            ctx->pair_first[p] = first_of_mol[m];
        }
    }
    if (prims.empty()) prims.push_back(PrimPair{});
    ctx->pairs = pairs;
    const int np = (int)pairs.size();
    PQB_CK(ctx, cudaMalloc(&ctx->d_pairs, sizeof(PairInfo) * np));
    PQB_CK(ctx, cudaMalloc(&ctx->d_prims, sizeof(PrimPair) * prims.size()));
    PQB_CK(ctx, cudaMalloc(&ctx->d_fscale, sizeof(double) * nbf));
    PQB_CK(ctx, cudaMalloc(&ctx->d_q2, sizeof(unsigned long long) * np));
    PQB_CK(ctx, cudaMemcpy(ctx->d_pairs, pairs.data(), sizeof(PairInfo) * np, cudaMemcpyHostToDevice));
    PQB_CK(ctx, cudaMemcpy(ctx->d_prims, prims.data(), sizeof(PrimPair) * prims.size(), cudaMemcpyHostToDevice));
    PQB_CK(ctx, cudaMemcpy(ctx->d_fscale, fscale, sizeof(double) * nbf, cudaMemcpyHostToDevice));
    {
        std::vector<int4> si(nshell);
        for (int sh = 0; sh < nshell; ++sh) {
            const int m = shell_mol[sh];
            si[sh] = make_int4(shell_f0[sh] - ctx->mol_f0[m], ncart(shell_l[sh]), m, 0);
        }
        PQB_CK(ctx, cudaMalloc(&ctx->d_shell_info, sizeof(int4) * nshell));
        PQB_CK(ctx, cudaMemcpy(ctx->d_shell_info, si.data(), sizeof(int4) * nshell, cudaMemcpyHostToDevice));
    }
    {
        std::vector<double> es((size_t)ctx->dense_len);
        for (int m = 0; m < nmol; ++m) {
            const int f0 = ctx->mol_f0[m], n = ctx->mol_n[m];
            for (int i = 0; i < n; ++i)
                for (int j = 0; j < n; ++j) es[(size_t)ctx->mol_off[m] + (size_t)i * n + j] = fscale[f0 + i] * fscale[f0 + j];
        }
        PQB_CK(ctx, cudaMalloc(&ctx->d_escale, sizeof(double) * std::max<size_t>(es.size(), 1)));
        PQB_CK(ctx, cudaMalloc(&ctx->d_Dscaled, sizeof(double) * std::max<size_t>(es.size(), 1)));
        PQB_CK(ctx, cudaMalloc(&ctx->d_Dscaled_f, sizeof(float) * std::max<size_t>(es.size(), 1)));
        PQB_CK(ctx, cudaMemcpy(ctx->d_escale, es.data(), sizeof(double) * es.size(), cudaMemcpyHostToDevice));
    }
    // unscreened quartet list (packed integrals) and diagonal list (Schwarz)
    std::vector<std::vector<int4>> dcls(kNumQuartetClass);
    for (int p = 0; p < np; ++p)
        dcls[quartet_class(pairs[p].cls, pairs[p].cls)].push_back(make_int4(p, p, 0, pairs[p].nprim * pairs[p].nprim));
    PQB_CK(ctx, cudaMalloc(&ctx->d_mol_off, sizeof(long long) * nmol));
    PQB_CK(ctx, cudaMalloc(&ctx->d_mol_n, sizeof(int) * nmol));
    PQB_CK(ctx, cudaMemcpy(ctx->d_mol_off, ctx->mol_off.data(), sizeof(long long) * nmol, cudaMemcpyHostToDevice));
    PQB_CK(ctx, cudaMemcpy(ctx->d_mol_n, ctx->mol_n.data(), sizeof(int) * nmol, cudaMemcpyHostToDevice));
    std::vector<int4> flat;
    bucket_sorted(dcls, flat, ctx->diag_off, ctx->diag_cnt);
    PQB_CK(ctx, cudaMalloc(&ctx->d_diag, sizeof(int4) * std::max<size_t>(flat.size(), 1)));
    PQB_CK(ctx, cudaMemcpy(ctx->d_diag, flat.data(), sizeof(int4) * flat.size(), cudaMemcpyHostToDevice));
    return PQB_OK;
}

int pqb_shells_upload_batch(pqb_ctx *ctx, int nmol, const int *mol_shell_off, int nshell, const int *shell_l,
                            const int *shell_nprim, const int *prim_off, const int *shell_f0, const double *shell_xyz,
                            const double *prim_exp, const double *prim_coef, int nbf, const double *fscale)
{
    try {
        return shells_upload_batch_impl(ctx, nmol, mol_shell_off, nshell, shell_l, shell_nprim, prim_off, shell_f0,
                                        shell_xyz, prim_exp, prim_coef, nbf, fscale);
    } catch (const std::bad_alloc &) {
        return fail(ctx, PQB_E_NOMEM, "pqb_shells_upload_batch: host allocation failed");
    } catch (...) {
        return fail(ctx, PQB_E_STATE, "pqb_shells_upload_batch: unexpected host exception");
    }
}

static int schwarz_impl(pqb_ctx *ctx, double *Q_host, void *stream)
{
    if (!ctx) return PQB_E_ARG;
    if (!ctx->d_pairs) return fail(ctx, PQB_E_STATE, "pqb_schwarz: no basis uploaded");
    PQB_CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    const int np = (int)ctx->pairs.size();
    PQB_CK(ctx, cudaMemsetAsync(ctx->d_q2, 0, sizeof(unsigned long long) * np, st));
    for (int c = 0; c < kNumQuartetClass; ++c)
        PQB_CK(ctx, launch_schwarz_f64(c, ctx->d_diag + ctx->diag_off[c], (int)ctx->diag_cnt[c], ctx->d_pairs,
                                       ctx->d_prims, ctx->d_q2, ctx->d_fscale, st, ctx->nsm));
    if (!ctx->d_Qpair) PQB_CK(ctx, cudaMalloc(&ctx->d_Qpair, sizeof(double) * np));
    double *dQ = ctx->d_Qpair;
    finalize_q_kernel<<<(np + 255) / 256, 256, 0, st>>>(ctx->d_q2, dQ, np);
    ctx->Q.assign(np, 0.0);
    cudaError_t e = cudaMemcpyAsync(ctx->Q.data(), dQ, sizeof(double) * np, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (ctx->scr.dmax) ctx->scr.Qpair = dQ;
    if (e != cudaSuccess) return fail(ctx, PQB_E_CUDA, "pqb_schwarz: %s", cudaGetErrorString(e));
    ctx->have_q = true;
    if (Q_host) memcpy(Q_host, ctx->Q.data(), sizeof(double) * np);
    return PQB_OK;
}

int pqb_schwarz(pqb_ctx *ctx, double *Q_host, void *stream)
{
    try {
        return schwarz_impl(ctx, Q_host, stream);
    } catch (const std::bad_alloc &) {
        return fail(ctx, PQB_E_NOMEM, "pqb_schwarz: host allocation failed");
    } catch (...) {
        return fail(ctx, PQB_E_STATE, "pqb_schwarz: unexpected host exception");
    }
}

int pqb_plan(pqb_ctx *ctx, double schwarz_thresh, double fp32_thresh, int64_t *counts)
{
    if (!ctx) return PQB_E_ARG;
    if (!ctx->have_q) return fail(ctx, PQB_E_STATE, "pqb_plan: call pqb_schwarz first");
    PQB_CK(ctx, cudaSetDevice(ctx->device));
    const auto &pairs = ctx->pairs;
    const auto &Q = ctx->Q;
    const int np = (int)pairs.size();
    // Enumeration: the bra pairs split into ranges of about equal quartet
    // counts, one per host thread; each range keeps its own per-class lists
    // in generation order, so the ranges in order are the sequential lists.
    std::vector<int64_t> cum(np + 1, 0);
    for (int p = 0; p < np; ++p) cum[p + 1] = cum[p] + (p - ctx->pair_first[p] + 1);
    const int64_t total = cum[np];
    const int T = ctx->plan_threads > 0 ? (int)std::min<int64_t>(ctx->plan_threads, std::max<int64_t>(np, 1))
                                        : (total < (int64_t)1 << 22 ? 1 : host_threads());
    std::vector<int> pb(T + 1, np);
    pb[0] = 0;
    for (int t = 1; t < T; ++t)
        pb[t] = std::max(pb[t - 1], (int)(std::lower_bound(cum.begin(), cum.end(), total * t / T) - cum.begin()));
    struct Range {
        std::vector<int4> items[2][kNumQuartetClass];
        int64_t prims[2][kNumQuartetClass] = {{0}};
        int64_t dropped = 0;
    };
    drop_graphs(ctx);
    ctx->have_plan = false;
    std::vector<Range> rg;
    try {
        rg.resize(T);
    } catch (...) {
        return fail(ctx, PQB_E_NOMEM, "pqb_plan: host allocation failed");
    }
    const bool enumerated = run_tasks(T, T, [&](int t) {
        Range &r = rg[t];
        for (int p = pb[t]; p < pb[t + 1]; ++p) {
            const int q0 = ctx->pair_first[p];
            for (int q = q0; q <= p; ++q) {
                const double b = Q[p] * Q[q];
                if (b < schwarz_thresh) {
                    ++r.dropped;
                    continue;
                }
                int qc;
                int4 e = oriented_quartet(pairs, p, q, qc);
                const int part = b < fp32_thresh ? 1 : 0;
                auto &dst = r.items[part][qc];
                const int ch = ctx->chunk[qc];
                for (int s0 = 0; s0 < e.w; s0 += ch) dst.push_back(make_int4(e.x, e.y, s0, std::min(ch, e.w - s0)));
                r.prims[part][qc] += e.w;
            }
        }
    });
    if (!enumerated) return fail(ctx, PQB_E_NOMEM, "pqb_plan: host allocation failed (quartet lists)");
    int64_t dropped = 0, nitems[2] = {0, 0};
    for (int t = 0; t < T; ++t) dropped += rg[t].dropped;
    for (int part = 0; part < 2; ++part)
        for (int c = 0; c < kNumQuartetClass; ++c) {
            int64_t n = 0, pr = 0;
            for (int t = 0; t < T; ++t) {
                n += (int64_t)rg[t].items[part][c].size();
                pr += rg[t].prims[part][c];
            }
            ctx->plan_cnt[part][c] = n;
            ctx->plan_prims[part][c] = pr;
            nitems[part] += n;
        }
    // class-major: the FP64 part of each class directly followed by its
    // FP32-eligible part, so an FP64 build launches one list per class
    int64_t o = 0;
    for (int c = 0; c < kNumQuartetClass; ++c)
        for (int part = 0; part < 2; ++part) {
            ctx->plan_off[part][c] = o;
            o += ctx->plan_cnt[part][c];
        }
    const size_t need = (size_t)o;
    try {
        ctx->plan_h.clear();
        ctx->plan_h.resize(need);
    } catch (...) {
        std::vector<int4>().swap(ctx->plan_h);
        return fail(ctx, PQB_E_NOMEM, "pqb_plan: host allocation failed (%zu work items)", need);
    }
    // Ordering: the (part, class) lists are independent; the largest go first
    std::vector<int> task(2 * kNumQuartetClass);
    for (int i = 0; i < 2 * kNumQuartetClass; ++i) task[i] = i;
    std::sort(task.begin(), task.end(), [&](int x, int y) {
        return ctx->plan_cnt[x / kNumQuartetClass][x % kNumQuartetClass] >
               ctx->plan_cnt[y / kNumQuartetClass][y % kNumQuartetClass];
    });
    const bool ordered = run_tasks(2 * kNumQuartetClass, T, [&](int i) {
        const int part = task[i] / kNumQuartetClass, c = task[i] % kNumQuartetClass;
        std::vector<const std::vector<int4> *> segs;
        for (int t = 0; t < T; ++t) segs.push_back(&rg[t].items[part][c]);
        order_class_items(segs, ctx->plan_h.data() + ctx->plan_off[part][c]);
        for (int t = 0; t < T; ++t) std::vector<int4>().swap(rg[t].items[part][c]);
    });
    if (!ordered) return fail(ctx, PQB_E_NOMEM, "pqb_plan: host allocation failed (ordering)");
    if (need > ctx->plan_cap) {
        free_dev(ctx->d_plan);
        ctx->d_plan = nullptr;
        PQB_CK(ctx, cudaMalloc(&ctx->d_plan, sizeof(int4) * std::max<size_t>(need, 1)));
        ctx->plan_cap = need;
    }
    if (need) PQB_CK(ctx, cudaMemcpy(ctx->d_plan, ctx->plan_h.data(), sizeof(int4) * need, cudaMemcpyHostToDevice));
    ctx->have_plan = true;
    if (counts) {
        counts[0] = total;
        counts[1] = nitems[0];
        counts[2] = nitems[1];
        counts[3] = dropped;
    }
    return PQB_OK;
}

int pqb_set_param(pqb_ctx *ctx, int param, int qclass, int value)
{
    if (!ctx) return PQB_E_ARG;
    drop_graphs(ctx);
    switch (param) {
    case PQB_PARAM_CHUNK:
        if (value < 1 || value > 4096) return fail(ctx, PQB_E_ARG, "chunk %d out of range 1..4096", value);
        if (qclass < 0) {
            for (int c = 0; c < kNumQuartetClass; ++c) ctx->chunk[c] = value;
        } else if (qclass < kNumQuartetClass) {
            ctx->chunk[qclass] = value;
        } else {
            return fail(ctx, PQB_E_ARG, "class %d", qclass);
        }
        ctx->have_plan = false;   // takes effect at the next pqb_plan
        return PQB_OK;
    case PQB_PARAM_STREAMS:
        if (value < 1 || value > pqb_ctx::kStreams) return fail(ctx, PQB_E_ARG, "streams %d out of range", value);
        ctx->nstreams = value;
        return PQB_OK;
    case PQB_PARAM_ORDER:
        if (value < 0 || value > 1) return fail(ctx, PQB_E_ARG, "order %d out of range", value);
        ctx->order = value;
        return PQB_OK;
    case PQB_PARAM_PACKED_KERNEL:
        if (value < 0 || value > 1) return fail(ctx, PQB_E_ARG, "packed kernel %d out of range", value);
        ctx->packed_simple = value == 1;
        return PQB_OK;
    case PQB_PARAM_GRAPH:
        if (value < 0 || value > 1) return fail(ctx, PQB_E_ARG, "graph %d out of range", value);
        ctx->use_graph = value == 1;
        return PQB_OK;
    case PQB_PARAM_THREADS:
        if (value < 0 || value > 256) return fail(ctx, PQB_E_ARG, "threads %d out of range 0..256", value);
        ctx->plan_threads = value;
        ctx->have_plan = false;   // takes effect at the next pqb_plan
        return PQB_OK;
    }
    return fail(ctx, PQB_E_ARG, "unknown parameter %d", param);
}

int pqb_plan_stats(const pqb_ctx *ctx, int64_t *quartets, int64_t *prim_quartets)
{
    if (!ctx || !quartets || !prim_quartets) return PQB_E_ARG;
    if (!ctx->have_plan) return PQB_E_STATE;
    for (int part = 0; part < 2; ++part)
        for (int c = 0; c < kNumQuartetClass; ++c) {
            quartets[part * kNumQuartetClass + c] = ctx->plan_cnt[part][c];
            prim_quartets[part * kNumQuartetClass + c] = ctx->plan_prims[part][c];
        }
    return PQB_OK;
}

static int plan_shard_impl(pqb_ctx *ctx, int rank, int nranks)
{
    if (!ctx || nranks < 1 || rank < 0 || rank >= nranks) return fail(ctx, PQB_E_ARG, "pqb_plan_shard: bad rank");
    if (!ctx->have_plan) return fail(ctx, PQB_E_STATE, "pqb_plan_shard: call pqb_plan first");
    if (nranks == 1) return PQB_OK;
    PQB_CK(ctx, cudaSetDevice(ctx->device));
    drop_graphs(ctx);
    const size_t total = ctx->plan_h.size();
    std::vector<int4> out;
    out.reserve(total / nranks + 64);
    int64_t off[2][kNumQuartetClass], cnt[2][kNumQuartetClass], prims[2][kNumQuartetClass];
    for (int c = 0; c < kNumQuartetClass; ++c)      // the class-major layout of pqb_plan
        for (int part = 0; part < 2; ++part) {
            off[part][c] = (int64_t)out.size();
            prims[part][c] = 0;
            for (int64_t q = rank; q < ctx->plan_cnt[part][c]; q += nranks) {
                const int4 e = ctx->plan_h[ctx->plan_off[part][c] + q];
                out.push_back(e);
                prims[part][c] += e.w;
            }
            cnt[part][c] = (int64_t)out.size() - off[part][c];
        }
    if (!out.empty())
        PQB_CK(ctx, cudaMemcpy(ctx->d_plan, out.data(), sizeof(int4) * out.size(), cudaMemcpyHostToDevice));
    memcpy(ctx->plan_off, off, sizeof off);
    memcpy(ctx->plan_cnt, cnt, sizeof cnt);
    memcpy(ctx->plan_prims, prims, sizeof prims);
    ctx->plan_h.swap(out);
    return PQB_OK;
}

int pqb_plan_shard(pqb_ctx *ctx, int rank, int nranks)
{
    try {
        return plan_shard_impl(ctx, rank, nranks);
    } catch (const std::bad_alloc &) {
        return fail(ctx, PQB_E_NOMEM, "pqb_plan_shard: host allocation failed");
    } catch (...) {
        return fail(ctx, PQB_E_STATE, "pqb_plan_shard: unexpected host exception");
    }
}

int pqb_fp64_peak(pqb_ctx *ctx, int iters, double *flops)
{
    if (!ctx || iters <= 0 || !flops) return fail(ctx, PQB_E_ARG, "pqb_fp64_peak: bad arguments");
    PQB_CK(ctx, cudaSetDevice(ctx->device));
    double *sink = nullptr;
    cudaEvent_t e0, e1;
    PQB_CK(ctx, cudaMalloc(&sink, sizeof(double)));
    PQB_CK(ctx, cudaEventCreate(&e0));
    PQB_CK(ctx, cudaEventCreate(&e1));
    const int blocks = ctx->nsm * 8, threads = 256;
    dfma_probe_kernel<<<blocks, threads>>>(iters / 10 + 1, sink);   // warm-up
    PQB_CK(ctx, cudaEventRecord(e0));
    dfma_probe_kernel<<<blocks, threads>>>(iters, sink);
    PQB_CK(ctx, cudaEventRecord(e1));
    PQB_CK(ctx, cudaEventSynchronize(e1));
    float ms = 0.f;
    PQB_CK(ctx, cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    *flops = 2.0 * 8.0 * (double)iters * blocks * threads / (ms * 1e-3);
    return PQB_OK;
}

// Unscreened list of every unique shell quartet (packed integrals), built
// on first use: P(P+1)/2 items, 16 bytes each.
static int ensure_full_list(pqb_ctx *ctx)
{
    if (ctx->d_full) return PQB_OK;
    const auto &pairs = ctx->pairs;
    const int np = (int)pairs.size();
    std::vector<std::vector<int4>> cls(kNumQuartetClass);
    for (int p = 0; p < np; ++p)
        for (int q = 0; q <= p; ++q) {
            int qc;
            int4 e = oriented_quartet(pairs, p, q, qc);
            cls[qc].push_back(e);
        }
    std::vector<int4> flat;
    bucket_sorted(cls, flat, ctx->full_off, ctx->full_cnt);
    PQB_CK(ctx, cudaMalloc(&ctx->d_full, sizeof(int4) * std::max<size_t>(flat.size(), 1)));
    PQB_CK(ctx, cudaMemcpy(ctx->d_full, flat.data(), sizeof(int4) * flat.size(), cudaMemcpyHostToDevice));
    return PQB_OK;
}

static int eri_packed_impl(pqb_ctx *ctx, double *out, int64_t len, void *stream)
{
    if (!ctx || !out) return fail(ctx, PQB_E_ARG, "pqb_eri_packed: bad arguments");
    if (!ctx->d_pairs) return fail(ctx, PQB_E_STATE, "pqb_eri_packed: no basis uploaded");
    if (ctx->nmol != 1) return fail(ctx, PQB_E_STATE, "pqb_eri_packed: batched basis (use pqb_jk_direct)");
    const int64_t P = (int64_t)ctx->nbf * (ctx->nbf + 1) / 2;
    if (len != P * (P + 1) / 2) return fail(ctx, PQB_E_SHAPE, "pqb_eri_packed: len %lld != %lld", (long long)len, (long long)(P * (P + 1) / 2));
    PQB_CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    {
        const int rc = ensure_full_list(ctx);
        if (rc != PQB_OK) return rc;
    }
    PQB_CK(ctx, ensure_streams(ctx));
    PQB_CK(ctx, cudaEventRecord(ctx->ev_fork, st));
    for (int k = 0; k < pqb_ctx::kStreams; ++k) PQB_CK(ctx, cudaStreamWaitEvent(ctx->streams[k], ctx->ev_fork, 0));
    for (int c = kNumQuartetClass - 1, k = 0; c >= 0; --c) {
        if (ctx->full_cnt[c] == 0) continue;
        PQB_CK(ctx, launch_packed_f64(c, ctx->d_full + ctx->full_off[c], (int)ctx->full_cnt[c], ctx->d_pairs,
                                      ctx->d_prims, out, ctx->d_fscale, ctx->streams[k++ % pqb_ctx::kStreams],
                                      ctx->nsm));
    }
    for (int k = 0; k < pqb_ctx::kStreams; ++k) {
        PQB_CK(ctx, cudaEventRecord(ctx->ev_join[k], ctx->streams[k]));
        PQB_CK(ctx, cudaStreamWaitEvent(st, ctx->ev_join[k], 0));
    }
    return PQB_OK;
}

int pqb_eri_packed(pqb_ctx *ctx, double *out, int64_t len, void *stream)
{
    try {
        return eri_packed_impl(ctx, out, len, stream);
    } catch (const std::bad_alloc &) {
        return fail(ctx, PQB_E_NOMEM, "pqb_eri_packed: host allocation failed");
    } catch (...) {
        return fail(ctx, PQB_E_STATE, "pqb_eri_packed: unexpected host exception");
    }
}

// The class launches of one build into the accumulators Jacc[s], Kacc[s]
// (zeroed here) of nden = 1 or 2 densities on stream st, forked over the
// context's streams and joined back; they read the scaled densities
// (d_Dscaled / d_Dscaled_f, and d_Dscaled2 / d_Dscaled2_f for the second).
// Kacc[0] == nullptr (one density): the Coulomb matrix alone.
// zero: clear the accumulators first (the graph's accumulators are kept
// zeroed by symmetrize_take_kernel instead).
static int launch_build(pqb_ctx *ctx, int nden, double *const Jacc[2], double *const Kacc[2], int mode,
                        cudaStream_t st, bool zero = true)
{
    const int n = ctx->nbf;
    const bool jonly = nden == 1 && !Kacc[0];
    for (int s = 0; s < nden && zero; ++s) {
        PQB_CK(ctx, cudaMemsetAsync(Jacc[s], 0, sizeof(double) * ctx->dense_len, st));
        if (!jonly) PQB_CK(ctx, cudaMemsetAsync(Kacc[s], 0, sizeof(double) * ctx->dense_len, st));
    }
    const double *Ds[2] = {ctx->d_Dscaled, ctx->d_Dscaled2};
    const float *Dsf[2] = {ctx->d_Dscaled_f, ctx->d_Dscaled2_f};
    const ItemScreen &mm = ctx->scr;
    // fork: class launches spread over the context's streams, heaviest first
    PQB_CK(ctx, cudaEventRecord(ctx->ev_fork, st));
    for (int k = 0; k < pqb_ctx::kStreams; ++k) PQB_CK(ctx, cudaStreamWaitEvent(ctx->streams[k], ctx->ev_fork, 0));
    int order[2 * kNumQuartetClass];
    double cost[2 * kNumQuartetClass];
    for (int i = 0; i < 2 * kNumQuartetClass; ++i) {
        order[i] = i;
        const int part = i / kNumQuartetClass, c = i % kNumQuartetClass;
        // order 1: classes with the longest per-item latency (high angular
        // momentum) start first so they do not form the tail of the build
        cost[i] = ctx->order == 1 ? (double)(c * 2 + (1 - part))
                                  : (double)ctx->plan_prims[part][c] * (1 + c) * (part == 1 && mode == PQB_MIXED ? 0.5 : 1.0);
    }
    std::sort(order, order + 2 * kNumQuartetClass, [&](int x, int y) { return cost[x] > cost[y]; });
    // in an FP64 build both parts of a class are one list (the plan is
    // class-major): one launch per class, over more items
    const bool merged = mode != PQB_MIXED;
    for (int i = 0, k = 0; i < 2 * kNumQuartetClass; ++i) {
        const int part = order[i] / kNumQuartetClass, c = order[i] % kNumQuartetClass;
        if (merged && part == 1) continue;
        const int nq = (int)(ctx->plan_cnt[part][c] + (merged ? ctx->plan_cnt[1][c] : 0));
        if (nq == 0) continue;
        cudaStream_t sk = ctx->streams[k++ % ctx->nstreams];
        const int4 *list = ctx->d_plan + ctx->plan_off[part][c];
        const bool f32 = part == 1 && mode == PQB_MIXED;
        if (jonly) {
            if (f32)
                PQB_CK(ctx, launch_j_f32(c, list, nq, ctx->d_pairs, ctx->d_prims, Ds[0], Dsf[0], Jacc[0], sk, ctx->nsm,
                                         mm));
            else
                PQB_CK(ctx, launch_j_f64(c, list, nq, ctx->d_pairs, ctx->d_prims, Ds[0], Jacc[0], sk, ctx->nsm, mm));
        } else if (nden == 2) {
            if (f32)
                PQB_CK(ctx, launch_jk2_f32(c, list, nq, ctx->d_pairs, ctx->d_prims, Ds, Dsf, Jacc, Kacc, sk, ctx->nsm,
                                           mm));
            else
                PQB_CK(ctx, launch_jk2_f64(c, list, nq, ctx->d_pairs, ctx->d_prims, Ds, Jacc, Kacc, sk, ctx->nsm, mm));
        } else if (f32) {
            PQB_CK(ctx, launch_jk_f32(c, list, nq, ctx->d_pairs, ctx->d_prims, Ds[0], Dsf[0], Jacc[0], Kacc[0], n, sk,
                                      ctx->nsm, mm));
        } else {
            PQB_CK(ctx, launch_jk_f64(c, list, nq, ctx->d_pairs, ctx->d_prims, Ds[0], Jacc[0], Kacc[0], n, sk,
                                      ctx->nsm, mm));
        }
    }
    // join
    for (int k = 0; k < pqb_ctx::kStreams; ++k) {
        PQB_CK(ctx, cudaEventRecord(ctx->ev_join[k], ctx->streams[k]));
        PQB_CK(ctx, cudaStreamWaitEvent(st, ctx->ev_join[k], 0));
    }
    return PQB_OK;
}

// Both accumulators of a pair or neither: a failed second allocation leaves
// no half-made pair behind.
static int ensure_acc_pair(pqb_ctx *ctx, double *&J, double *&K)
{
    if (J && K) return PQB_OK;
    free_dev(J);
    free_dev(K);
    J = K = nullptr;
    const size_t bytes = sizeof(double) * std::max<long long>(ctx->dense_len, 1);
    cudaError_t e = cudaMalloc(&J, bytes);
    if (e == cudaSuccess) e = cudaMalloc(&K, bytes);
    // zeroed once here; each use leaves them zeroed (symmetrize_take_kernel)
    if (e == cudaSuccess) e = cudaMemset(J, 0, bytes);
    if (e == cudaSuccess) e = cudaMemset(K, 0, bytes);
    if (e != cudaSuccess) {
        free_dev(J);
        free_dev(K);
        J = K = nullptr;
        return fail(ctx, PQB_E_CUDA, "graph accumulators: %s", cudaGetErrorString(e));
    }
    return PQB_OK;
}

// Capture launch_build into the ctx-owned accumulators as a graph for
// (nden, mode) (index gi), once; later builds replay it with one launch.
static int ensure_build_graph(pqb_ctx *ctx, int nden, bool jonly, int mode, int gi)
{
    if (ctx->graph_exec[gi]) return PQB_OK;
    if (!ctx->cap_stream) PQB_CK(ctx, cudaStreamCreateWithFlags(&ctx->cap_stream, cudaStreamNonBlocking));
    int rc = ensure_acc_pair(ctx, ctx->d_Jacc, ctx->d_Kacc);
    if (rc == PQB_OK && nden == 2) rc = ensure_acc_pair(ctx, ctx->d_Jacc2, ctx->d_Kacc2);
    if (rc != PQB_OK) return rc;
    double *const Ja[2] = {ctx->d_Jacc, ctx->d_Jacc2};
    double *const Ka[2] = {jonly ? nullptr : ctx->d_Kacc, ctx->d_Kacc2};
    PQB_CK(ctx, cudaStreamBeginCapture(ctx->cap_stream, cudaStreamCaptureModeThreadLocal));
    rc = launch_build(ctx, nden, Ja, Ka, mode, ctx->cap_stream, false);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(ctx->cap_stream, &g);   // always ends the capture
    if (rc != PQB_OK || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return rc != PQB_OK ? rc : fail(ctx, PQB_E_CUDA, "graph capture: %s", cudaGetErrorString(e));
    }
    const cudaError_t ei = cudaGraphInstantiate(&ctx->graph_exec[gi], g, 0);
    cudaGraphDestroy(g);
    if (ei != cudaSuccess) {
        ctx->graph_exec[gi] = nullptr;
        return fail(ctx, PQB_E_CUDA, "graph instantiate: %s", cudaGetErrorString(ei));
    }
    return PQB_OK;
}

// J and K of nden densities D[s] into J[s], K[s] (K[0] == nullptr with one
// density: J alone).
// J and K of nden densities.  With G (one density, J and K wanted): G = 2J - K
// as well; on the graph path G alone is written (J, K untouched), else J and
// K are written and then combined.
static int jk_direct_impl(pqb_ctx *ctx, int nden, const double *const D[2], double *const J[2], double *const K[2],
                          int mode, void *stream, double *G = nullptr)
{
    const bool jonly = nden == 1 && !K[0];
    const int n = ctx->nbf;
    cudaStream_t st = (cudaStream_t)stream;
    PQB_CK(ctx, ensure_streams(ctx));
    if (nden == 2 && !ctx->d_Dscaled2) {
        const size_t len = std::max<long long>(ctx->dense_len, 1);
        PQB_CK(ctx, cudaMalloc(&ctx->d_Dscaled2, sizeof(double) * len));
        const cudaError_t e = cudaMalloc(&ctx->d_Dscaled2_f, sizeof(float) * len);
        if (e != cudaSuccess) {
            free_dev(ctx->d_Dscaled2);
            ctx->d_Dscaled2 = nullptr;
            ctx->d_Dscaled2_f = nullptr;
            return fail(ctx, PQB_E_CUDA, "second scaled density: %s", cudaGetErrorString(e));
        }
    }
    double *Dsc[2] = {ctx->d_Dscaled, ctx->d_Dscaled2};
    float *Dsf[2] = {ctx->d_Dscaled_f, ctx->d_Dscaled2_f};
    for (int s = 0; s < nden; ++s)
        scale_elements_kernel<<<ctx->nsm * 4, 256, 0, st>>>(D[s], ctx->d_escale, Dsc[s], Dsf[s], ctx->dense_len);
    const int64_t P = (int64_t)n * (n + 1) / 2;
    // graph replay for a single molecule when the caller is not capturing
    // (a caller's own capture records the launches themselves)
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    PQB_CK(ctx, cudaStreamIsCapturing(st, &cs));
    const int gi = (jonly ? 4 : (nden == 2 ? 2 : 0)) + (mode == PQB_MIXED ? 1 : 0);
    if (ctx->use_graph && ctx->nmol == 1 && cs == cudaStreamCaptureStatusNone && ctx->graph_warm[gi]) {
        const int rc = ensure_build_graph(ctx, nden, jonly, mode, gi);
        if (rc != PQB_OK) return rc;
        PQB_CK(ctx, cudaGraphLaunch(ctx->graph_exec[gi], st));
        double *Ja[2] = {ctx->d_Jacc, ctx->d_Jacc2}, *Ka[2] = {ctx->d_Kacc, ctx->d_Kacc2};
        if (G) {
            take_2jmk_kernel<<<(unsigned)((P + 255) / 256), 256, 0, st>>>(Ja[0], Ka[0], G, n, ctx->d_escale);
            PQB_CK(ctx, cudaGetLastError());
            return PQB_OK;
        }
        for (int s = 0; s < nden; ++s)
            symmetrize_take_kernel<<<(unsigned)((P + 255) / 256), 256, 0, st>>>(
                Ja[s], J[s], jonly ? nullptr : Ka[s], jonly ? nullptr : K[s], n, ctx->d_escale);
        PQB_CK(ctx, cudaGetLastError());
        return PQB_OK;
    }
    const int rc = launch_build(ctx, nden, J, K, mode, st);
    if (rc != PQB_OK) return rc;
    if (cs == cudaStreamCaptureStatusNone) ctx->graph_warm[gi] = true;
    for (int s = 0; s < nden; ++s) {
        if (ctx->nmol == 1) {
            symmetrize_kernel<<<(unsigned)((P + 255) / 256), 256, 0, st>>>(J[s], n, ctx->d_escale);
            if (!jonly) symmetrize_kernel<<<(unsigned)((P + 255) / 256), 256, 0, st>>>(K[s], n, ctx->d_escale);
        } else {
            symmetrize_blocks_kernel<<<ctx->nmol, 256, 0, st>>>(J[s], ctx->d_mol_off, ctx->d_mol_n, ctx->d_escale);
            if (!jonly)
                symmetrize_blocks_kernel<<<ctx->nmol, 256, 0, st>>>(K[s], ctx->d_mol_off, ctx->d_mol_n, ctx->d_escale);
        }
    }
    if (G) combine_2jmk_kernel<<<ctx->nsm * 4, 256, 0, st>>>(J[0], K[0], G, (int64_t)n * n);
    PQB_CK(ctx, cudaGetLastError());
    return PQB_OK;
}

int pqb_jk_direct(pqb_ctx *ctx, const double *D, double *J, double *K, int mode, void *stream)
{
    if (!ctx || !D || !J) return fail(ctx, PQB_E_ARG, "pqb_jk_direct: bad arguments");
    if (!ctx->have_plan) return fail(ctx, PQB_E_STATE, "pqb_jk_direct: call pqb_plan first");
    if (mode != PQB_FP64 && mode != PQB_MIXED) return fail(ctx, PQB_E_ARG, "pqb_jk_direct: mode %d", mode);
    PQB_CK(ctx, cudaSetDevice(ctx->device));
    const double *Dv[2] = {D, nullptr};
    double *Jv[2] = {J, nullptr}, *Kv[2] = {K, nullptr};
    return jk_direct_impl(ctx, 1, Dv, Jv, Kv, mode, stream);
}

static int get2jmk_host_impl(pqb_ctx *ctx, const double *D_host, double *G_host, int mode, void *stream)
{
    if (!ctx || !D_host || !G_host) return fail(ctx, PQB_E_ARG, "pqb_get2jmk_host: bad arguments");
    if (!ctx->have_plan) return fail(ctx, PQB_E_STATE, "pqb_get2jmk_host: call pqb_plan first");
    if (ctx->nmol != 1) return fail(ctx, PQB_E_STATE, "pqb_get2jmk_host: one molecule per context");
    if (mode != PQB_FP64 && mode != PQB_MIXED) return fail(ctx, PQB_E_ARG, "pqb_get2jmk_host: mode %d", mode);
    PQB_CK(ctx, cudaSetDevice(ctx->device));
    const int n = ctx->nbf;
    const size_t bytes = sizeof(double) * (size_t)n * n;
    double **bufs[4] = {&ctx->d_hD, &ctx->d_hG, &ctx->d_hJ, &ctx->d_hK};
    for (double **b : bufs)
        if (!*b) PQB_CK(ctx, cudaMalloc(b, bytes));
    cudaStream_t st = (cudaStream_t)stream;
    PQB_CK(ctx, cudaMemcpyAsync(ctx->d_hD, D_host, bytes, cudaMemcpyHostToDevice, st));
    const double *Dv[2] = {ctx->d_hD, nullptr};
    double *Jv[2] = {ctx->d_hJ, nullptr}, *Kv[2] = {ctx->d_hK, nullptr};
    const int rc = jk_direct_impl(ctx, 1, Dv, Jv, Kv, mode, stream, ctx->d_hG);
    if (rc != PQB_OK) return rc;
    PQB_CK(ctx, cudaMemcpyAsync(G_host, ctx->d_hG, bytes, cudaMemcpyDeviceToHost, st));
    return PQB_OK;
}

int pqb_get2jmk_host(pqb_ctx *ctx, const double *D_host, double *G_host, int mode, void *stream)
{
    try {
        return get2jmk_host_impl(ctx, D_host, G_host, mode, stream);
    } catch (const std::bad_alloc &) {
        return fail(ctx, PQB_E_NOMEM, "pqb_get2jmk_host: host allocation failed");
    } catch (...) {
        return fail(ctx, PQB_E_STATE, "pqb_get2jmk_host: unexpected host exception");
    }
}

int pqb_jk_direct2(pqb_ctx *ctx, const double *Da, const double *Db, double *Ja, double *Ka, double *Jb, double *Kb,
                   int mode, void *stream)
{
    if (!ctx || !Da || !Db || !Ja || !Ka || !Jb || !Kb) return fail(ctx, PQB_E_ARG, "pqb_jk_direct2: bad arguments");
    if (!ctx->have_plan) return fail(ctx, PQB_E_STATE, "pqb_jk_direct2: call pqb_plan first");
    if (mode != PQB_FP64 && mode != PQB_MIXED) return fail(ctx, PQB_E_ARG, "pqb_jk_direct2: mode %d", mode);
    PQB_CK(ctx, cudaSetDevice(ctx->device));
    const double *Dv[2] = {Da, Db};
    double *Jv[2] = {Ja, Jb}, *Kv[2] = {Ka, Kb};
    return jk_direct_impl(ctx, 2, Dv, Jv, Kv, mode, stream);
}

int pqb_set_molecule_mask(pqb_ctx *ctx, const int *mask)
{
    if (!ctx) return PQB_E_ARG;
    ctx->scr.molmask = mask;
    drop_graphs(ctx);   // a captured build holds the old screen
    return PQB_OK;
}

int pqb_set_density_screen(pqb_ctx *ctx, const double *shell_dmax, double tau)
{
    if (!ctx || tau < 0.0) return fail(ctx, PQB_E_ARG, "pqb_set_density_screen: bad arguments");
    if (shell_dmax && !ctx->d_Qpair)
        return fail(ctx, PQB_E_STATE, "pqb_set_density_screen: call pqb_schwarz (or pqb_plan) first");
    ctx->scr.dmax = shell_dmax;
    ctx->scr.Qpair = shell_dmax ? ctx->d_Qpair : nullptr;
    ctx->scr.tau = tau;
    drop_graphs(ctx);
    return PQB_OK;
}

int pqb_shell_dmax(pqb_ctx *ctx, const double *D, double *shell_dmax, void *stream)
{
    if (!ctx || !D || !shell_dmax) return fail(ctx, PQB_E_ARG, "pqb_shell_dmax: bad arguments");
    if (!ctx->d_shell_info) return fail(ctx, PQB_E_STATE, "pqb_shell_dmax: no basis uploaded");
    PQB_CK(ctx, cudaSetDevice(ctx->device));
    const int warps = 8;
    shell_dmax_kernel<<<(ctx->nshell + warps - 1) / warps, warps * 32, 0, (cudaStream_t)stream>>>(
        ctx->nshell, ctx->d_shell_info, ctx->d_mol_off, ctx->d_mol_n, D, shell_dmax);
    PQB_CK(ctx, cudaGetLastError());
    return PQB_OK;
}

int pqb_dense_len(const pqb_ctx *ctx, int64_t *len)
{
    if (!ctx || !len) return PQB_E_ARG;
    *len = ctx->dense_len;
    return PQB_OK;
}

int pqb_jk_direct_class(pqb_ctx *ctx, const double *D, double *Jacc, double *Kacc, int part, int qclass, int mode,
                        void *stream)
{
    if (!ctx || !D || !Jacc || !Kacc || part < 0 || part > 1 || qclass < 0 || qclass >= kNumQuartetClass)
        return fail(ctx, PQB_E_ARG, "pqb_jk_direct_class: bad arguments");
    if (!ctx->have_plan) return fail(ctx, PQB_E_STATE, "pqb_jk_direct_class: call pqb_plan first");
    PQB_CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    const int4 *list = ctx->d_plan + ctx->plan_off[part][qclass];
    const int nq = (int)ctx->plan_cnt[part][qclass];
    scale_elements_kernel<<<ctx->nsm * 4, 256, 0, st>>>(D, ctx->d_escale, ctx->d_Dscaled, ctx->d_Dscaled_f,
                                                         ctx->dense_len);
    if (mode == PQB_MIXED && part == 1)
        PQB_CK(ctx, launch_jk_f32(qclass, list, nq, ctx->d_pairs, ctx->d_prims, ctx->d_Dscaled, ctx->d_Dscaled_f, Jacc,
                                  Kacc, ctx->nbf, st, ctx->nsm));
    else
        PQB_CK(ctx, launch_jk_f64(qclass, list, nq, ctx->d_pairs, ctx->d_prims, ctx->d_Dscaled, Jacc, Kacc, ctx->nbf,
                                  st, ctx->nsm));
    return PQB_OK;
}

static int jk_packed_impl(pqb_ctx *ctx, const double *ints, int64_t len, const double *D, double *J, double *K, int nbf,
                          void *stream)
{
    if (!ctx || !ints || !D || !J || !K || nbf <= 0) return fail(ctx, PQB_E_ARG, "pqb_jk_packed: bad arguments");
    const int64_t P = (int64_t)nbf * (nbf + 1) / 2;
    if (len != P * (P + 1) / 2) return fail(ctx, PQB_E_SHAPE, "pqb_jk_packed: len %lld != %lld", (long long)len, (long long)(P * (P + 1) / 2));
    if (P > 0x7fffffffLL) return fail(ctx, PQB_E_SHAPE, "pqb_jk_packed: nbf too large");
    PQB_CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    PQB_CK(ctx, cudaMemsetAsync(J, 0, sizeof(double) * nbf * nbf, st));
    PQB_CK(ctx, cudaMemsetAsync(K, 0, sizeof(double) * nbf * nbf, st));
    if (nbf <= 512 && !ctx->packed_simple) {
        // register form: tiles (i, j0) of 16 rows, heaviest (largest i) first
        if (ctx->pk_tiles_nbf != nbf) {
            std::vector<int2> tiles;
            for (int i = nbf - 1; i >= 0; --i)
                for (int j0 = 0; j0 <= i; j0 += kRgRows) tiles.push_back(make_int2(i, j0));
            free_dev(ctx->d_pk_tiles);
            ctx->d_pk_tiles = nullptr;
            PQB_CK(ctx, cudaMalloc(&ctx->d_pk_tiles, sizeof(int2) * tiles.size()));
            PQB_CK(ctx, cudaMemcpy(ctx->d_pk_tiles, tiles.data(), sizeof(int2) * tiles.size(), cudaMemcpyHostToDevice));
            ctx->pk_tiles_n = (int)tiles.size();
            ctx->pk_tiles_nbf = nbf;
        }
        int grid = ctx->pk_tiles_n;
        if (grid > ctx->nsm * 16) grid = ctx->nsm * 16;
        // register rows sized to the column count: 32 * MAXM >= nbf
        const int need = (nbf + 31) / 32;
        const int2 *tl = ctx->d_pk_tiles;
        const int nt = ctx->pk_tiles_n;
        if (need <= 2) PQB_CK(ctx, launch_packed_reg<2>(ints, D, J, K, nbf, tl, nt, grid, st));
        else if (need <= 4) PQB_CK(ctx, launch_packed_reg<4>(ints, D, J, K, nbf, tl, nt, grid, st));
        else if (need <= 6) PQB_CK(ctx, launch_packed_reg<6>(ints, D, J, K, nbf, tl, nt, grid, st));
        else if (need <= 7) PQB_CK(ctx, launch_packed_reg<7>(ints, D, J, K, nbf, tl, nt, grid, st));
        else if (need <= 8) PQB_CK(ctx, launch_packed_reg<8>(ints, D, J, K, nbf, tl, nt, grid, st));
        else if (need <= 10) PQB_CK(ctx, launch_packed_reg<10>(ints, D, J, K, nbf, tl, nt, grid, st));
        else if (need <= 12) PQB_CK(ctx, launch_packed_reg<12>(ints, D, J, K, nbf, tl, nt, grid, st));
        else PQB_CK(ctx, launch_packed_reg<16>(ints, D, J, K, nbf, tl, nt, grid, st));
    } else {
        // one block per packed row (nbf > 512: the packed array alone is then over 69 GB)
        jk_packed_kernel<<<(unsigned)P, 256, 0, st>>>(ints, D, J, K, nbf);
    }
    symmetrize_kernel<<<(unsigned)((P + 255) / 256), 256, 0, st>>>(J, nbf, nullptr);
    symmetrize_kernel<<<(unsigned)((P + 255) / 256), 256, 0, st>>>(K, nbf, nullptr);
    PQB_CK(ctx, cudaGetLastError());
    return PQB_OK;
}

int pqb_jk_packed(pqb_ctx *ctx, const double *ints, int64_t len, const double *D, double *J, double *K, int nbf,
                  void *stream)
{
    try {
        return jk_packed_impl(ctx, ints, len, D, J, K, nbf, stream);
    } catch (const std::bad_alloc &) {
        return fail(ctx, PQB_E_NOMEM, "pqb_jk_packed: host allocation failed");
    } catch (...) {
        return fail(ctx, PQB_E_STATE, "pqb_jk_packed: unexpected host exception");
    }
}

static int eri_functions_impl(pqb_ctx *ctx, int engine, int aux_m, int nq, const int *quartets, int n, const double *origin,
                              const int *powers, const int *prim_off, const double *exps, const double *cn,
                              const double *norms, double *out, void *stream)
{
    if (!ctx || nq < 0 || !quartets || n <= 0 || !origin || !powers || !prim_off || !exps || !cn || !norms || !out)
        return fail(ctx, PQB_E_ARG, "pqb_eri_functions: bad arguments");
    if (engine != PQB_ENGINE_RYS && engine != PQB_ENGINE_HGP)
        return fail(ctx, PQB_E_ARG, "pqb_eri_functions: engine %d", engine);
    if (aux_m < 0 || (aux_m > 0 && engine != PQB_ENGINE_HGP))
        return fail(ctx, PQB_E_ARG, "pqb_eri_functions: aux_m %d needs the HGP engine", aux_m);
    if (nq == 0) return PQB_OK;
    PQB_CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    FuncTable ft{origin, powers, prim_off, exps, cn, norms};
    if (engine == PQB_ENGINE_RYS)
        eri_general_rys_kernel<<<(nq + 63) / 64, 64, 0, st>>>(nq, quartets, ft, out);
    else
        eri_general_hgp_kernel<<<(nq + 31) / 32, 32, 0, st>>>(nq, aux_m, quartets, ft, out);
    PQB_CK(ctx, cudaGetLastError());
    return PQB_OK;
}

int pqb_eri_functions(pqb_ctx *ctx, int engine, int aux_m, int nq, const int *quartets, int n, const double *origin,
                      const int *powers, const int *prim_off, const double *exps, const double *cn,
                      const double *norms, double *out, void *stream)
{
    try {
        return eri_functions_impl(ctx, engine, aux_m, nq, quartets, n, origin, powers, prim_off, exps, cn, norms, out,
                                  stream);
    } catch (const std::bad_alloc &) {
        return fail(ctx, PQB_E_NOMEM, "pqb_eri_functions: host allocation failed");
    } catch (...) {
        return fail(ctx, PQB_E_STATE, "pqb_eri_functions: unexpected host exception");
    }
}

static int oneint_impl(pqb_ctx *ctx, int n, const double *origin, const int *powers, const int *prim_off, const double *exps,
                       const double *cn, const double *norms, int natoms, const double *atom_xyz, const double *atom_z,
                       double *S, double *T, double *V, void *stream)
{
    if (!ctx || n <= 0 || !origin || !powers || !prim_off || !exps || !cn || !norms || natoms < 0 ||
        (V && natoms > 0 && (!atom_xyz || !atom_z)))
        return fail(ctx, PQB_E_ARG, "pqb_oneint: bad arguments");
    PQB_CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    // atoms (host arrays) -> packed device scratch {x, y, z, Z}
    std::vector<double> at(4 * (size_t)std::max(natoms, 1), 0.0);
    for (int a = 0; a < natoms; ++a) {
        for (int x = 0; x < 3; ++x) at[4 * a + x] = atom_xyz[3 * a + x];
        at[4 * a + 3] = atom_z[a];
    }
    if (at.size() > ctx->atoms_cap) {
        free_dev(ctx->d_atoms);
        ctx->d_atoms = nullptr;
        PQB_CK(ctx, cudaMalloc(&ctx->d_atoms, sizeof(double) * at.size()));
        ctx->atoms_cap = at.size();
    }
    PQB_CK(ctx, cudaMemcpyAsync(ctx->d_atoms, at.data(), sizeof(double) * at.size(), cudaMemcpyHostToDevice, st));
    FuncTable ft{origin, powers, prim_off, exps, cn, norms};
    const int64_t nn = (int64_t)n * n;
    oneint_kernel<<<(unsigned)((nn + 127) / 128), 128, 0, st>>>(n, ft, natoms, ctx->d_atoms, S, T, V);
    PQB_CK(ctx, cudaGetLastError());
    // the host staging buffer must outlive the async copy
    PQB_CK(ctx, cudaStreamSynchronize(st));
    return PQB_OK;
}

int pqb_oneint(pqb_ctx *ctx, int n, const double *origin, const int *powers, const int *prim_off, const double *exps,
               const double *cn, const double *norms, int natoms, const double *atom_xyz, const double *atom_z,
               double *S, double *T, double *V, void *stream)
{
    try {
        return oneint_impl(ctx, n, origin, powers, prim_off, exps, cn, norms, natoms, atom_xyz, atom_z, S, T, V,
                           stream);
    } catch (const std::bad_alloc &) {
        return fail(ctx, PQB_E_NOMEM, "pqb_oneint: host allocation failed");
    } catch (...) {
        return fail(ctx, PQB_E_STATE, "pqb_oneint: unexpected host exception");
    }
}

// Host code may not use pqb_noalloc_atoms' name as a device address: its
// device address is looked up once per device with cudaGetSymbolAddress
// (with that device current) and cached here.
static double *g_noalloc_atoms[PQB_NOALLOC_MAX_DEVICES] = {nullptr};
static std::mutex g_noalloc_mutex;

int pqb_oneint_noalloc(int n, const double *origin, const int *powers, const int *prim_off, const double *exps,
                       const double *cn, const double *norms, int natoms, const double *atom_xyz,
                       const double *atom_z, double *S, double *T, double *V, void *stream)
{
    // the same argument rules as pqb_oneint: atoms are read only for V
    if (n <= 0 || !origin || !powers || !prim_off || !exps || !cn || !norms || natoms < 0 ||
        (V && natoms > 0 && (!atom_xyz || !atom_z)))
        return PQB_E_ARG;
    if (natoms > PQB_NOALLOC_MAX_ATOMS) return PQB_E_SHAPE;
    // a non-sticky error left by an unrelated earlier call must not be read
    // as this call's launch status below
    (void)cudaGetLastError();
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= PQB_NOALLOC_MAX_DEVICES) return PQB_E_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    // the scratch address below is the current device's copy: a stream of
    // another device would launch against the wrong one
    int sdev = dev;
    if (cudaStreamGetDevice(st, &sdev) != cudaSuccess) return PQB_E_CUDA;
    if (sdev != dev) return PQB_E_ARG;
    const int nat = V ? natoms : 0;
    double *atoms = nullptr;
    if (nat > 0) {
        std::lock_guard<std::mutex> lock(g_noalloc_mutex);
        if (!g_noalloc_atoms[dev]) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, pqb_noalloc_atoms) != cudaSuccess || !p) return PQB_E_CUDA;
            g_noalloc_atoms[dev] = static_cast<double *>(p);
        }
        atoms = g_noalloc_atoms[dev];
        pack_atoms_kernel<<<(nat + 127) / 128, 128, 0, st>>>(nat, atom_xyz, atom_z, atoms);
    }
    FuncTable ft{origin, powers, prim_off, exps, cn, norms};
    const int64_t nn = (int64_t)n * n;
    oneint_kernel<<<(unsigned)((nn + 127) / 128), 128, 0, st>>>(n, ft, nat, atoms, S, T, V);
    return cudaGetLastError() == cudaSuccess ? PQB_OK : PQB_E_CUDA;
}

static int set_shell_atoms_impl(pqb_ctx *ctx, const int *shell_atom)
{
    if (!ctx || !shell_atom) return fail(ctx, PQB_E_ARG, "pqb_set_shell_atoms: bad arguments");
    if (!ctx->d_pairs) return fail(ctx, PQB_E_STATE, "pqb_set_shell_atoms: no basis uploaded");
    PQB_CK(ctx, cudaSetDevice(ctx->device));
    if (!ctx->d_shell_atom) PQB_CK(ctx, cudaMalloc(&ctx->d_shell_atom, sizeof(int) * ctx->nshell));
    PQB_CK(ctx, cudaMemcpy(ctx->d_shell_atom, shell_atom, sizeof(int) * ctx->nshell, cudaMemcpyHostToDevice));
    return PQB_OK;
}

int pqb_set_shell_atoms(pqb_ctx *ctx, const int *shell_atom)
{
    try {
        return set_shell_atoms_impl(ctx, shell_atom);
    } catch (const std::bad_alloc &) {
        return fail(ctx, PQB_E_NOMEM, "pqb_set_shell_atoms: host allocation failed");
    } catch (...) {
        return fail(ctx, PQB_E_STATE, "pqb_set_shell_atoms: unexpected host exception");
    }
}

static int grad_2e_impl(pqb_ctx *ctx, const double *D, double *grad, int mode, void *stream)
{
    if (!ctx || !D || !grad) return fail(ctx, PQB_E_ARG, "pqb_grad_2e: bad arguments");
    if (!ctx->have_plan) return fail(ctx, PQB_E_STATE, "pqb_grad_2e: call pqb_plan first");
    if (!ctx->d_shell_atom) return fail(ctx, PQB_E_STATE, "pqb_grad_2e: call pqb_set_shell_atoms first");
    PQB_CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    for (int part = 0; part < 2; ++part)
        for (int c = 0; c < kNumQuartetClass; ++c) {
            const int nq = (int)ctx->plan_cnt[part][c];
            if (nq == 0) continue;
            const int4 *list = ctx->d_plan + ctx->plan_off[part][c];
            if (part == 1 && mode == PQB_MIXED)
                PQB_CK(ctx, launch_grad_f32(c, list, nq, ctx->d_pairs, ctx->d_prims, D, ctx->d_fscale,
                                            ctx->d_shell_atom, ctx->nbf, grad, st, ctx->nsm));
            else
                PQB_CK(ctx, launch_grad_f64(c, list, nq, ctx->d_pairs, ctx->d_prims, D, ctx->d_fscale,
                                            ctx->d_shell_atom, ctx->nbf, grad, st, ctx->nsm));
        }
    return PQB_OK;
}

int pqb_grad_2e(pqb_ctx *ctx, const double *D, double *grad, int mode, void *stream)
{
    try {
        return grad_2e_impl(ctx, D, grad, mode, stream);
    } catch (const std::bad_alloc &) {
        return fail(ctx, PQB_E_NOMEM, "pqb_grad_2e: host allocation failed");
    } catch (...) {
        return fail(ctx, PQB_E_STATE, "pqb_grad_2e: unexpected host exception");
    }
}

static int grad_1e_impl(pqb_ctx *ctx, int n, const double *origin, const int *powers, const int *prim_off, const double *exps,
                        const double *cn, const double *norms, const int *func_atom, int natoms, const double *atom_xyz,
                        const double *atom_z, const double *D, const double *W, double *grad, void *stream)
{
    if (!ctx || n <= 0 || !origin || !powers || !prim_off || !exps || !cn || !norms || !func_atom || natoms <= 0 ||
        !atom_xyz || !atom_z || !D || !W || !grad)
        return fail(ctx, PQB_E_ARG, "pqb_grad_1e: bad arguments");
    PQB_CK(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    std::vector<double> at(4 * (size_t)natoms);
    for (int a = 0; a < natoms; ++a) {
        for (int x = 0; x < 3; ++x) at[4 * a + x] = atom_xyz[3 * a + x];
        at[4 * a + 3] = atom_z[a];
    }
    if (at.size() > ctx->atoms_cap) {
        free_dev(ctx->d_atoms);
        ctx->d_atoms = nullptr;
        PQB_CK(ctx, cudaMalloc(&ctx->d_atoms, sizeof(double) * at.size()));
        ctx->atoms_cap = at.size();
    }
    PQB_CK(ctx, cudaMemcpyAsync(ctx->d_atoms, at.data(), sizeof(double) * at.size(), cudaMemcpyHostToDevice, st));
    FuncTable ft{origin, powers, prim_off, exps, cn, norms};
    const int64_t nn = (int64_t)n * n;
    oneint_grad_kernel<<<(unsigned)((nn + 127) / 128), 128, 0, st>>>(n, ft, natoms, ctx->d_atoms, func_atom, D, W,
                                                                     grad);
    PQB_CK(ctx, cudaGetLastError());
    PQB_CK(ctx, cudaStreamSynchronize(st));
    return PQB_OK;
}

int pqb_grad_1e(pqb_ctx *ctx, int n, const double *origin, const int *powers, const int *prim_off, const double *exps,
                const double *cn, const double *norms, const int *func_atom, int natoms, const double *atom_xyz,
                const double *atom_z, const double *D, const double *W, double *grad, void *stream)
{
    try {
        return grad_1e_impl(ctx, n, origin, powers, prim_off, exps, cn, norms, func_atom, natoms, atom_xyz, atom_z, D,
                            W, grad, stream);
    } catch (const std::bad_alloc &) {
        return fail(ctx, PQB_E_NOMEM, "pqb_grad_1e: host allocation failed");
    } catch (...) {
        return fail(ctx, PQB_E_STATE, "pqb_grad_1e: unexpected host exception");
    }
}

int pqb_boys_eval(pqb_ctx *ctx, int m, int count, const double *T, double *F, void *stream)
{
    if (!ctx || m < 0 || m > 16 || count < 0 || !T || !F) return fail(ctx, PQB_E_ARG, "pqb_boys_eval: bad arguments");
    if (count == 0) return PQB_OK;
    PQB_CK(ctx, cudaSetDevice(ctx->device));
    boys_eval_kernel<<<(count + 127) / 128, 128, 0, (cudaStream_t)stream>>>(m, count, T, F);
    PQB_CK(ctx, cudaGetLastError());
    return PQB_OK;
}

int pqb_boys_rows_eval(pqb_ctx *ctx, int lt, int count, const double *T, double *F, void *stream)
{
    if (!ctx || lt < 0 || lt > 4 || count < 0 || !T || !F) return fail(ctx, PQB_E_ARG, "pqb_boys_rows_eval: bad arguments");
    if (count == 0) return PQB_OK;
    PQB_CK(ctx, cudaSetDevice(ctx->device));
    boys_rows_eval_kernel<<<(count + 127) / 128, 128, 0, (cudaStream_t)stream>>>(lt, count, T, F);
    PQB_CK(ctx, cudaGetLastError());
    return PQB_OK;
}

int pqb_rys_eval(pqb_ctx *ctx, int nroots, int count, const double *T, double *u, double *w, void *stream)
{
    if (!ctx || nroots < 1 || nroots > PQB_RYS_NMAX || count < 0 || !T || !u || !w)
        return fail(ctx, PQB_E_ARG, "pqb_rys_eval: bad arguments");
    if (count == 0) return PQB_OK;
    PQB_CK(ctx, cudaSetDevice(ctx->device));
    rys_eval_kernel<<<(count + 127) / 128, 128, 0, (cudaStream_t)stream>>>(nroots, count, T, u, w);
    PQB_CK(ctx, cudaGetLastError());
    return PQB_OK;
}

}  // extern "C"
