// Shell-quartet ERI engine: one kernel template per angular-momentum class
// (LA LB | LC LD), fed a class-sorted list of (bra pair, ket pair) quartets.
//
// Two integral schemes, chosen per class at compile time:
//  * classes with LA+LB+LC+LD <= 4 (thread mode): the Obara--Saika vertical
//    recurrence per primitive quartet and the Head-Gordon--Pople horizontal
//    transfer once per contracted item (the scheme of the reference's
//    Src/chgp.c:78-419), as straight-line code generated by gen_os.py
//    (os_classes.inc);
//  * the rest: the Rys quadrature of the reference's Src/crys.c:56-97 (sum
//    over roots of Ix*Iy*Iz*w, ABD eqs 5, 9).
// Both are organised per SHELL quartet: the recurrences run once per
// primitive quartet and serve every cartesian component, instead of once per
// component as crys.contr_coulomb does (Src/crys.c:34-54).
//
// Two execution modes:
//  * thread mode (NAB*NCD <= 81, which is every class with L <= 4): one
//    thread per work item; the recurrence intermediates and all contracted
//    components live in registers.
//  * block mode (larger classes): a 256-thread block holds NSQ = 256/NAB
//    quartets; per primitive quartet the roots (NSQ*NR tasks) and the 2-D
//    integrals (NSQ*NR*3 tasks) go to shared memory, then every thread
//    accumulates the NCD ket components of one bra component pair in
//    registers.
//
// The epilogue functor consumes the contracted integrals of one bra
// component pair (ia, ib) for all ket components, so the same engine
// writes packed integrals, digests into J/K, or forms Schwarz bounds.
#pragma once
#include <atomic>
#include <type_traits>
#include "pqb_device.cuh"
#include "pqb_types.h"

namespace pqb {

struct QCtx {
    int fa, fb, fc, fd;   // first function index of the four shells
    int sa, sb, sc, sd;   // shell indices
    int bra, ket;         // pair ids (bra == ket: diagonal quartet)
    int nm;               // row length of the molecule's D/J/K block
    long long bo;         // element (i, j) of that block: bo + i*nm + j
};

__device__ __forceinline__ QCtx make_qctx(const PairInfo &pb, const PairInfo &pk, int bra, int ket)
{
    return QCtx{pb.fa, pb.fb, pk.fa, pk.fb, pb.sa, pb.sb, pk.sa, pk.sb, bra, ket, pb.nm, pb.bo};
}

__device__ __forceinline__ int64_t fpair(int i, int j)
{
    return i >= j ? (int64_t)i * (i + 1) / 2 + j : (int64_t)j * (j + 1) / 2 + i;
}

// ------------------------------------------------------------ epilogues --
// Every epilogue offers
//   thread_quartet<LA,LB,LC,LD>(q, acc[NAB*NCD], lane, live)
//                                                  whole quartet, thread mode (all lanes
//                                                  of the warp call it; live = a real item)
//   kTile                                          false: block mode calls
//     block_ab<LA,LB,LC,LD>(q, ia, ib, acc[NCD])     per bra component pair;
//                                                  true: block mode stores the
//     tile_store<LA,LB,LC,LD>(q, ia, ib, acc, V)     quartet's weighted integrals
//     tile_reduce<LA,LB,LC,LD>(q, V, t, nt)          in a shared tile V and reduces
//                                                    them after a block barrier

__device__ __forceinline__ bool skip_bra(const QCtx &q, int fi, int fj) { return q.sa == q.sb && fi < fj; }

// 1 if (x0, y0) > (x1, y1) lexicographically, 1/2 if equal, 0 if less.
__host__ __device__ constexpr double lex_weight(int x0, int y0, int x1, int y1)
{
    return x0 != x1 ? (x0 > x1 ? 1.0 : 0.0) : (y0 != y1 ? (y0 > y1 ? 1.0 : 0.0) : 0.5);
}

// Degeneracy weight of component (ia ib|ic id) of a unique shell quartet:
// 0 outside the canonical ranges i >= j, k >= l, ij >= kl; a factor 1/2 for
// each of i == j, k == l, ij == kl; else 1.  Only the flags are runtime:
//   bd: the bra's two shells are one shell (then i - j = ia - ib),
//   kd: the same for the ket,
//   qd: bra pair == ket pair (then IJ vs KL orders (ia, ib) vs (ic, id)
//       lexicographically when the first shell holds the higher function
//       indices, af, or bd; otherwise (ib, ia) vs (id, ic)).
// In the unrolled loops the component indices are constants, so each weight
// is a few selects: no branches and no 64-bit pair indices per component.
__device__ __forceinline__ double comp_weight(int ia, int ib, int ic, int id, bool bd, bool kd, bool qd, bool af)
{
    const double wb = ia > ib ? 1.0 : (ia == ib ? 0.5 : 0.0);
    const double wk = ic > id ? 1.0 : (ic == id ? 0.5 : 0.0);
    const double wq = (bd || af) ? lex_weight(ia, ib, ic, id) : lex_weight(ib, ia, id, ic);
    return (bd ? wb : 1.0) * (kd ? wk : 1.0) * (qd ? wq : 1.0);
}

// Packed canonical integrals at ijkl2intindex (Src/cints.c:413-425), 64-bit.
struct EpiPacked {
    double *out;
    const double *fscale;
    static constexpr bool kTile = false;
    __device__ __forceinline__ bool screened(const PairInfo &, const PairInfo &, int, int) const { return false; }
    template <int LC, int LD, typename R>
    __device__ __forceinline__ void ab(const QCtx &q, int ia, int ib, const R *acc) const
    {
        constexpr int NC = ncart(LC), ND = ncart(LD);
        const int fi = q.fa + ia, fj = q.fb + ib;
        if (skip_bra(q, fi, fj)) return;
        const int64_t IJ = fpair(fi, fj);
        const double sij = fscale[fi] * fscale[fj];
#pragma unroll
        for (int ic = 0; ic < NC; ++ic)
#pragma unroll
            for (int id = 0; id < ND; ++id) {
                const int fk = q.fc + ic, fl = q.fd + id;
                if (q.sc == q.sd && fk < fl) continue;
                const int64_t KL = fpair(fk, fl);
                if (q.bra == q.ket && IJ < KL) continue;
                const int64_t hi = IJ > KL ? IJ : KL, lo = IJ > KL ? KL : IJ;
                out[hi * (hi + 1) / 2 + lo] = (double)acc[ic * ND + id] * sij * fscale[fk] * fscale[fl];
            }
    }
    template <int LA, int LB, int LC, int LD, typename R>
    __device__ __forceinline__ void thread_quartet(const QCtx &q, const R *acc, int lane, bool live) const
    {
        constexpr int NB = ncart(LB), NCD = ncart(LC) * ncart(LD);
        (void)lane;
        if (!live) return;
#pragma unroll
        for (int ab = 0; ab < ncart(LA) * NB; ++ab) this->ab<LC, LD, R>(q, ab / NB, ab % NB, acc + ab * NCD);
    }
    template <int LA, int LB, int LC, int LD, typename R>
    __device__ __forceinline__ void block_ab(const QCtx &q, int ia, int ib, const R *acc) const
    {
        ab<LC, LD, R>(q, ia, ib, acc);
    }
};

// Runs of equal keys over the lanes of a warp (the thread-mode item lists
// are ordered so that neighbouring lanes often share a bra pair and a ket
// shell): sum() is an inclusive segmented scan, so the last lane of a run
// holds the run's total and issues one atomic for the whole run.  Every lane
// of the warp must take part.
struct WarpRuns {
    unsigned f;   // bit s: lane - 2^s lies in this lane's run
    bool last;    // last lane of its run
    __device__ __forceinline__ WarpRuns(long long key, int lane)
    {
        // a run is a maximal block of consecutive lanes with one key (the
        // same key may come back later in the warp as another run): first
        // the lane where this lane's run starts (max-scan of run heads)
        const long long kp = __shfl_up_sync(0xffffffffu, key, 1);
        int start = (lane == 0 || kp != key) ? lane : 0;
#pragma unroll
        for (int s = 0; s < 5; ++s) {
            const int o = __shfl_up_sync(0xffffffffu, start, 1 << s);
            if (lane >= (1 << s) && o > start) start = o;
        }
        f = 0;
#pragma unroll
        for (int s = 0; s < 5; ++s)
            if (lane - (1 << s) >= start) f |= 1u << s;
        const long long kn = __shfl_down_sync(0xffffffffu, key, 1);
        last = lane == 31 || kn != key;
    }
    template <typename V> __device__ __forceinline__ V sum(V x) const
    {
#pragma unroll
        for (int s = 0; s < 5; ++s) {
            const V y = __shfl_up_sync(0xffffffffu, x, 1 << s);
            if ((f >> s) & 1u) x += y;
        }
        return x;
    }
};

// Full-warp sums of K values per lane (K <= 32) by recursive halving: at each
// of the first log2(KP) butterfly levels (KP = K rounded up to a power of two)
// every lane keeps half of its remaining values and adds its partner's half
// of them, then the remaining levels are a plain butterfly.  Lane L ends with
// the warp's sum of value idx(L) (the kept halves), held by the 32/KP lanes
// that agree on those bits; (KP - 1) + (5 - log2 KP) shuffles in place of the
// 5 K of K separate sums.  Every lane of the warp must take part.
template <int K, typename V>
__device__ __forceinline__ V warp_sum_transposed(const V *v, int lane, int &idx)
{
    constexpr int KP = K <= 1 ? 1 : K <= 2 ? 2 : K <= 4 ? 4 : K <= 8 ? 8 : K <= 16 ? 16 : 32;
    V w[KP];
#pragma unroll
    for (int j = 0; j < KP; ++j) w[j] = j < K ? v[j] : (V)0;
    idx = 0;
    int o = 16;
#pragma unroll
    for (int n = KP; n > 1; n >>= 1, o >>= 1) {
        const bool up = (lane & o) != 0;
#pragma unroll
        for (int j = 0; j < n / 2; ++j) {
            const V keep = up ? w[j + n / 2] : w[j], send = up ? w[j] : w[j + n / 2];
            w[j] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
        if (up) idx += n / 2;
    }
#pragma unroll
    for (; o > 0; o >>= 1) w[0] += __shfl_xor_sync(0xffffffffu, w[0], o);
    return w[0];
}

// Direct J/K digestion of unique quartets with 8-fold degeneracy weights:
//   Jacc[i,j] += 2 v' D_kl,  Jacc[k,l] += 2 v' D_ij,
//   Kacc[i,k] += v' D_jl, Kacc[i,l] += v' D_jk, Kacc[j,k] += v' D_il, Kacc[j,l] += v' D_ik,
// v' = v * comp_weight; then J = Jacc + Jacc^T, K = Kacc + Kacc^T reproduce
// J_ij = sum_kl (ij|kl) D_kl and K_ij = sum_kl (ik|jl) D_kl of
// PyQuante/Ints.py:195-223 for symmetric D.
//
// The integrals here are those of the shells' common contraction (no
// per-component scale r_f): D is the pre-scaled density D'_kl = r_k r_l D_kl
// and the caller multiplies J and K by r_i r_j afterwards, which gives the
// same J and K as digesting the scaled integrals with D.
//
// Thread mode: the quartet's six D blocks are loaded once, the six J/K
// blocks (ab, cd, ac, ad, bc, bd) are summed in registers, and each block
// element goes to global memory with one atomic.  Block mode: the weighted
// integrals go to a shared tile; each output element is then one thread's
// reduction over the tile (no shared-memory atomics).  With NDEN = 2 both
// densities are digested from the same integrals (UHF); WITHK = false keeps
// the Coulomb terms alone.
template <int NDEN, bool WITHK = true>
struct EpiJKn {
    const double *D[NDEN];        // pre-scaled densities
    double *Jacc[NDEN], *Kacc[NDEN];
    const float *Df[NDEN];        // their single-precision copies (FP32 lists of the mixed mode), or null
    ItemScreen scr;               // items skipped by molecule mask or density bound (all fields optional)
    static constexpr bool kTile = true;
    __device__ __forceinline__ bool screened(const PairInfo &pb, const PairInfo &pk, int bra, int ket) const
    {
        if (scr.molmask && __ldg(scr.molmask + pb.mol) == 0) return true;
        if (scr.dmax) {
            const double d = fmax(fmax(__ldg(scr.dmax + pb.sa), __ldg(scr.dmax + pb.sb)),
                                  fmax(__ldg(scr.dmax + pk.sa), __ldg(scr.dmax + pk.sb)));
            if (__ldg(scr.Qpair + bra) * __ldg(scr.Qpair + ket) * d < scr.tau) return true;
        }
        return false;
    }

    // (called by every lane of the warp; a lane past the end of the item list
    // passes its neighbour's quartet with zero integrals)
    // The per-quartet products, block sums and sums over lanes run in the
    // list's precision R (FP32 lists read the single-precision density); the
    // accumulation into Jacc/Kacc is FP64.
    template <int LA, int LB, int LC, int LD, typename R>
    __device__ __forceinline__ void thread_quartet(const QCtx &q, const R *acc, int lane, bool) const
    {
        using T = R;
        constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD), NCD = NC * ND;
        const bool bd = q.sa == q.sb, kd = q.sc == q.sd, qd = q.bra == q.ket, af = q.fa > q.fb;
        // Jacc[a,b] is shared by lanes with the same bra pair; Kacc[a,c] and
        // Kacc[b,c] by lanes that also share the ket's first shell (the bra
        // runs are scanned only for warps of more than one bra pair)
        const WarpRuns rbc(((long long)q.bra << 32) | (unsigned)q.sc, lane);
        // (the shuffle is taken by every lane, outside any condition)
        const int bra0 = __shfl_sync(0xffffffffu, q.bra, 0);
        const bool one_bra = __all_sync(0xffffffffu, bra0 == q.bra);
        // every density digests the same integrals, one after the other
#pragma unroll
        for (int s = 0; s < NDEN; ++s) {
        const T *Db;
        if constexpr (std::is_same_v<T, float>)
            Db = Df[s] + q.bo;
        else
            Db = D[s] + q.bo;
        double *Jb = Jacc[s] + q.bo, *Kb = Kacc[s] + q.bo;
        const int64_t nm = q.nm;
        const T *Da = Db + q.fa * nm, *Dbr = Db + q.fb * nm, *Dc = Db + q.fc * nm;
        // Coulomb: Jacc[a,b] and Jacc[c,d]
        {
            T dab[NA][NB], dcd[NC][ND], jcd[NC][ND];
#pragma unroll
            for (int a = 0; a < NA; ++a)
#pragma unroll
                for (int b = 0; b < NB; ++b) dab[a][b] = __ldg(Da + a * nm + q.fb + b);
#pragma unroll
            for (int c = 0; c < NC; ++c)
#pragma unroll
                for (int d = 0; d < ND; ++d) {
                    dcd[c][d] = __ldg(Dc + c * nm + q.fd + d);
                    jcd[c][d] = (T)0;
                }
            T jabv[NA * NB];
#pragma unroll
            for (int a = 0; a < NA; ++a)
#pragma unroll
                for (int b = 0; b < NB; ++b) {
                    T jab = (T)0;
#pragma unroll
                    for (int c = 0; c < NC; ++c)
#pragma unroll
                        for (int d = 0; d < ND; ++d) {
                            const T v = (T)acc[(a * NB + b) * NCD + c * ND + d] *
                                        (T)comp_weight(a, b, c, d, bd, kd, qd, af);
                            jab = fma(v, dcd[c][d], jab);
                            jcd[c][d] = fma(v, dab[a][b], jcd[c][d]);
                        }
                    jabv[a * NB + b] = jab;
                }
            if (NA * NB <= 32 && one_bra) {
                // the whole warp is one bra pair: all NAB sums in one transposed reduction
                int idx;
                const double js = (double)warp_sum_transposed<(NA * NB <= 32 ? NA * NB : 1)>(jabv, lane, idx);
                constexpr int KP = NA * NB <= 1 ? 1 : NA * NB <= 2 ? 2 : NA * NB <= 4 ? 4 : NA * NB <= 8 ? 8 : NA * NB <= 16 ? 16 : 32;
                if (idx < NA * NB && (lane & (32 / KP - 1)) == 0 && js != 0.0)
                    atomicAdd(Jb + (q.fa + idx / NB) * nm + q.fb + idx % NB, 2.0 * js);
            } else {
                const WarpRuns rb((long long)q.bra, lane);
#pragma unroll
                for (int ab = 0; ab < NA * NB; ++ab) {
                    const double js = (double)rb.sum(jabv[ab]);
                    if (rb.last && js != 0.0) atomicAdd(Jb + (q.fa + ab / NB) * nm + q.fb + ab % NB, 2.0 * js);
                }
            }
#pragma unroll
            for (int c = 0; c < NC; ++c)
#pragma unroll
                for (int d = 0; d < ND; ++d)
                    if (jcd[c][d] != (T)0) atomicAdd(Jb + (q.fc + c) * nm + q.fd + d, 2.0 * (double)jcd[c][d]);
        }
        if constexpr (!WITHK) continue;   // Coulomb only
        // exchange rows of the bra's first shell: Kacc[a,c] += v D_bd, Kacc[a,d] += v D_bc
        {
            T dbd[NB][ND], dbc[NB][NC];
#pragma unroll
            for (int b = 0; b < NB; ++b) {
#pragma unroll
                for (int d = 0; d < ND; ++d) dbd[b][d] = __ldg(Dbr + b * nm + q.fd + d);
#pragma unroll
                for (int c = 0; c < NC; ++c) dbc[b][c] = __ldg(Dbr + b * nm + q.fc + c);
            }
#pragma unroll
            for (int a = 0; a < NA; ++a) {
                T kac[NC], kad[ND];
#pragma unroll
                for (int c = 0; c < NC; ++c) kac[c] = (T)0;
#pragma unroll
                for (int d = 0; d < ND; ++d) kad[d] = (T)0;
#pragma unroll
                for (int b = 0; b < NB; ++b)
#pragma unroll
                    for (int c = 0; c < NC; ++c)
#pragma unroll
                        for (int d = 0; d < ND; ++d) {
                            const T v = (T)acc[(a * NB + b) * NCD + c * ND + d] *
                                        (T)comp_weight(a, b, c, d, bd, kd, qd, af);
                            kac[c] = fma(v, dbd[b][d], kac[c]);
                            kad[d] = fma(v, dbc[b][c], kad[d]);
                        }
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    const double ks = (double)rbc.sum(kac[c]);
                    if (rbc.last && ks != 0.0) atomicAdd(Kb + (q.fa + a) * nm + q.fc + c, ks);
                }
#pragma unroll
                for (int d = 0; d < ND; ++d)
                    if (kad[d] != (T)0) atomicAdd(Kb + (q.fa + a) * nm + q.fd + d, (double)kad[d]);
            }
        }
        // exchange rows of the bra's second shell: Kacc[b,c] += v D_ad, Kacc[b,d] += v D_ac
        {
            T dad[NA][ND], dac[NA][NC];
#pragma unroll
            for (int a = 0; a < NA; ++a) {
#pragma unroll
                for (int d = 0; d < ND; ++d) dad[a][d] = __ldg(Da + a * nm + q.fd + d);
#pragma unroll
                for (int c = 0; c < NC; ++c) dac[a][c] = __ldg(Da + a * nm + q.fc + c);
            }
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                T kbc[NC], kbd[ND];
#pragma unroll
                for (int c = 0; c < NC; ++c) kbc[c] = (T)0;
#pragma unroll
                for (int d = 0; d < ND; ++d) kbd[d] = (T)0;
#pragma unroll
                for (int a = 0; a < NA; ++a)
#pragma unroll
                    for (int c = 0; c < NC; ++c)
#pragma unroll
                        for (int d = 0; d < ND; ++d) {
                            const T v = (T)acc[(a * NB + b) * NCD + c * ND + d] *
                                        (T)comp_weight(a, b, c, d, bd, kd, qd, af);
                            kbc[c] = fma(v, dad[a][d], kbc[c]);
                            kbd[d] = fma(v, dac[a][c], kbd[d]);
                        }
#pragma unroll
                for (int c = 0; c < NC; ++c) {
                    const double ks = (double)rbc.sum(kbc[c]);
                    if (rbc.last && ks != 0.0) atomicAdd(Kb + (q.fb + b) * nm + q.fc + c, ks);
                }
#pragma unroll
                for (int d = 0; d < ND; ++d)
                    if (kbd[d] != (T)0) atomicAdd(Kb + (q.fb + b) * nm + q.fd + d, (double)kbd[d]);
            }
        }
        }
    }

    // block mode: the tile row of bra component (ia, ib) holds its NCD
    // weighted integrals (row stride NCD + 1 spreads the rows over the banks)
    template <int LA, int LB, int LC, int LD>
    static constexpr int kTileStride = ncart(LC) * ncart(LD) + 1;

    template <int LA, int LB, int LC, int LD, typename R>
    __device__ __forceinline__ void tile_store(const QCtx &q, int ia, int ib, const R *acc, double *V) const
    {
        constexpr int NC = ncart(LC), ND = ncart(LD), NB = ncart(LB);
        constexpr int ST = kTileStride<LA, LB, LC, LD>;
        const bool bd = q.sa == q.sb, kd = q.sc == q.sd, qd = q.bra == q.ket, af = q.fa > q.fb;
        const int64_t nm = q.nm;
        // runtime bra indices: the bra and quartet factors of comp_weight in closed form
        const double wb = bd ? (ia > ib ? 1.0 : (ia == ib ? 0.5 : 0.0)) : 1.0;
        const int x0 = (bd || af) ? ia : ib, y0 = (bd || af) ? ib : ia;
        double jab[NDEN];
#pragma unroll
        for (int s = 0; s < NDEN; ++s) jab[s] = 0.0;
        double *row = V + (ia * NB + ib) * ST;
#pragma unroll
        for (int c = 0; c < NC; ++c)
#pragma unroll
            for (int d = 0; d < ND; ++d) {
                const double wk = kd ? (c > d ? 1.0 : (c == d ? 0.5 : 0.0)) : 1.0;
                const int x1 = (bd || af) ? c : d, y1 = (bd || af) ? d : c;
                const double wq = qd ? (x0 != x1 ? (x0 > x1 ? 1.0 : 0.0) : (y0 != y1 ? (y0 > y1 ? 1.0 : 0.0) : 0.5))
                                     : 1.0;
                const double v = (double)acc[c * ND + d] * (wb * wk * wq);
#pragma unroll
                for (int s = 0; s < NDEN; ++s) jab[s] = fma(v, __ldg(D[s] + q.bo + (q.fc + c) * nm + q.fd + d), jab[s]);
                row[c * ND + d] = v;
            }
#pragma unroll
        for (int s = 0; s < NDEN; ++s)
            if (jab[s] != 0.0) atomicAdd(Jacc[s] + q.bo + (q.fa + ia) * nm + q.fb + ib, 2.0 * jab[s]);
    }

    // outputs of one quartet: Jacc[c,d] (NCD), Kacc[a,c], Kacc[a,d],
    // Kacc[b,c], Kacc[b,d]; threads t, t + nt, ... of the quartet's slot
    template <int LA, int LB, int LC, int LD>
    __device__ __forceinline__ void tile_reduce(const QCtx &q, const double *V, int t, int nt) const
    {
        constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD), NCD = NC * ND;
        constexpr int ST = kTileStride<LA, LB, LC, LD>;
        constexpr int O1 = NCD, O2 = O1 + NA * NC, O3 = O2 + NA * ND, O4 = O3 + NB * NC,
                      O5 = WITHK ? O4 + NB * ND : O1;
        const int64_t nm = q.nm;
#pragma unroll
        for (int sd = 0; sd < NDEN; ++sd) {
        const double *Db = D[sd] + q.bo;
        double *Jo = Jacc[sd], *Ko = Kacc[sd];
        for (int o = t; o < O5; o += nt) {
            double s = 0.0;
            double *dst;
            if (o < O1) {                     // Jacc[c,d] = 2 sum_ab v D_ab
                const int c = o / ND, d = o - (o / ND) * ND;
                for (int a = 0; a < NA; ++a)
                    for (int b = 0; b < NB; ++b)
                        s = fma(V[(a * NB + b) * ST + c * ND + d], __ldg(Db + (q.fa + a) * nm + q.fb + b), s);
                s *= 2.0;
                dst = Jo + q.bo + (q.fc + c) * nm + q.fd + d;
            } else if (o < O2) {              // Kacc[a,c] = sum_bd v D_bd
                const int a = (o - O1) / NC, c = (o - O1) - ((o - O1) / NC) * NC;
                for (int b = 0; b < NB; ++b)
                    for (int d = 0; d < ND; ++d)
                        s = fma(V[(a * NB + b) * ST + c * ND + d], __ldg(Db + (q.fb + b) * nm + q.fd + d), s);
                dst = Ko + q.bo + (q.fa + a) * nm + q.fc + c;
            } else if (o < O3) {              // Kacc[a,d] = sum_bc v D_bc
                const int a = (o - O2) / ND, d = (o - O2) - ((o - O2) / ND) * ND;
                for (int b = 0; b < NB; ++b)
                    for (int c = 0; c < NC; ++c)
                        s = fma(V[(a * NB + b) * ST + c * ND + d], __ldg(Db + (q.fb + b) * nm + q.fc + c), s);
                dst = Ko + q.bo + (q.fa + a) * nm + q.fd + d;
            } else if (o < O4) {              // Kacc[b,c] = sum_ad v D_ad
                const int b = (o - O3) / NC, c = (o - O3) - ((o - O3) / NC) * NC;
                for (int a = 0; a < NA; ++a)
                    for (int d = 0; d < ND; ++d)
                        s = fma(V[(a * NB + b) * ST + c * ND + d], __ldg(Db + (q.fa + a) * nm + q.fd + d), s);
                dst = Ko + q.bo + (q.fb + b) * nm + q.fc + c;
            } else {                          // Kacc[b,d] = sum_ac v D_ac
                const int b = (o - O4) / ND, d = (o - O4) - ((o - O4) / ND) * ND;
                for (int a = 0; a < NA; ++a)
                    for (int c = 0; c < NC; ++c)
                        s = fma(V[(a * NB + b) * ST + c * ND + d], __ldg(Db + (q.fa + a) * nm + q.fc + c), s);
                dst = Ko + q.bo + (q.fb + b) * nm + q.fd + d;
            }
            if (s != 0.0) atomicAdd(dst, s);
        }
        }
    }
};

// One density (RHF, or one spin at a time) and two (UHF's alpha and beta
// densities digesting the same integrals in one pass).
using EpiJK = EpiJKn<1>;
using EpiJK2 = EpiJKn<2>;
// Coulomb only (DFT's getJ): no exchange products, no K atomics
using EpiJ = EpiJKn<1, false>;



// Schwarz: Q2[pair] = max over components of |(ij|ij)| (diagonal quartets).
struct EpiSchwarz {
    unsigned long long *Q2bits;   // bit patterns of non-negative doubles
    const double *fscale;
    static constexpr bool kTile = false;
    __device__ __forceinline__ bool screened(const PairInfo &, const PairInfo &, int, int) const { return false; }
    template <int LC, int LD, typename R>
    __device__ __forceinline__ void ab(const QCtx &q, int ia, int ib, const R *acc) const
    {
        constexpr int ND = ncart(LD), NCD = ncart(LC) * ncart(LD);
        const int cd = ia * ND + ib;   // (ic, id) == (ia, ib) on a diagonal quartet
        double v = 0.0;
#pragma unroll
        for (int c = 0; c < NCD; ++c)
            if (c == cd) v = (double)acc[c];
        const double s = fscale[q.fa + ia] * fscale[q.fb + ib];
        v = fabs(v) * s * s;
        atomicMax(Q2bits + q.bra, (unsigned long long)__double_as_longlong(v));
    }
    template <int LA, int LB, int LC, int LD, typename R>
    __device__ __forceinline__ void thread_quartet(const QCtx &q, const R *acc, int lane, bool live) const
    {
        constexpr int NB = ncart(LB), NCD = ncart(LC) * ncart(LD);
        (void)lane;
        if (!live) return;
#pragma unroll
        for (int ab = 0; ab < ncart(LA) * NB; ++ab) this->ab<LC, LD, R>(q, ab / NB, ab % NB, acc + ab * NCD);
    }
    template <int LA, int LB, int LC, int LD, typename R>
    __device__ __forceinline__ void block_ab(const QCtx &q, int ia, int ib, const R *acc) const
    {
        ab<LC, LD, R>(q, ia, ib, acc);
    }
};

// ------------------------------------------------- Obara--Saika classes --
// Per-primitive-quartet coefficients of the Obara--Saika vertical recurrence
// (PA = P - A, QC = Q - C, WP = -rho/zeta PQ, WQ = rho/eta PQ, PQ = P - Q,
// rz = rho/zeta = eta/(zeta+eta), re = rho/eta = zeta/(zeta+eta),
// oo2z = 1/(2 zeta), oo2e = 1/(2 eta), oo2ze = 1/(2 (zeta+eta))).
template <typename R>
struct OsGeom {
    R PA[3], WP[3], QC[3], WQ[3];
    R oo2z, rz, oo2e, re, oo2ze;
};

// Classes without generated routines keep the Rys quadrature.
template <int LA, int LB, int LC, int LD>
struct OsClass {
    static constexpr bool kOn = false;
    static constexpr int NV = 1;
    template <typename R>
    __device__ static void vrr(const OsGeom<R> &, const R *, R *) {}
    template <typename R>
    __device__ static void hrr(const R *, const R *, const R *, R *) {}
};

#include "os_classes.inc"

// ---------------------------------------------------------- thread mode --
// Register cap per class (via the minimum resident blocks of 128 threads):
// small classes are latency bound, so they trade registers for occupancy
// (six blocks for up to three components, five for up to nine, three for
// the 27 of (11|10), measured faster than fewer even with a few spilled
// registers).
__host__ __device__ constexpr int thread_min_blocks(int nabcd)
{
    return nabcd == 1 ? 8 : (nabcd <= 3 ? 6 : (nabcd <= 9 ? 5 : (nabcd == 27 ? 3 : 2)));
}

// Single-precision counterpart of add_prim_quartet for the FP32 lists of
// the mixed mode: geometry, roots (rys_roots_f32), 2-D tables and assembly
// all in FP32; only large-T root forms are evaluated in FP64.
struct QuartetGeomF {
    float A[3], C[3], AB[3], CD[3];
};

template <int LA, int LB, int LC, int LD>
__device__ __forceinline__ void add_prim_quartet_f32(const QuartetGeomF &g, const float *P, const float *Q, float *acc)
{
    constexpr int NB = ncart(LB), ND = ncart(LD);
    constexpr int NAB = ncart(LA) * NB, NCD = ncart(LC) * ND;
    constexpr int NR = (LA + LB + LC + LD) / 2 + 1;
    constexpr int G2D = (LA + 1) * (LB + 1) * (LC + 1) * (LD + 1);
    // P, Q: zeta, 1/zeta, P[3], K
    const float zeta = P[0], eta = Q[0];
    const float PQ[3] = {P[2] - Q[2], P[3] - Q[3], P[4] - Q[4]};
    const float rs = rsqrtf(zeta + eta), izpe = rs * rs;
    const float T = zeta * eta * izpe * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
    const float pre = P[5] * Q[5] * rs;
    float uu[NR], ww[NR];
    rys_roots_f32<NR>(T, uu, ww);
#pragma unroll
    for (int r = 0; r < NR; ++r) {
        const float ue = uu[r] * izpe, ce = eta * ue, cz = zeta * ue;
        const float b00 = 0.5f * ue, b10 = 0.5f * P[1] * (1.0f - ce), b01 = 0.5f * Q[1] * (1.0f - cz);
        float gx[G2D], gy[G2D], gz[G2D];
        float *gt[3] = {gx, gy, gz};
#pragma unroll
        for (int x = 0; x < 3; ++x)
            rys2d_f<LA, LB, LC, LD>(b00, b10, b01, fmaf(-ce, PQ[x], P[2 + x] - g.A[x]), fmaf(cz, PQ[x], Q[2 + x] - g.C[x]),
                                    g.AB[x], g.CD[x], x == 0 ? ww[r] * pre : 1.0f, gt[x]);
#pragma unroll
        for (int ab = 0; ab < NAB; ++ab)
#pragma unroll
            for (int cd = 0; cd < NCD; ++cd) {
                const int ia = ab / NB, ib = ab % NB, ic = cd / ND, id = cd % ND;
                const int ox = ((cart_lx(LA, ia) * (LB + 1) + cart_lx(LB, ib)) * (LC + 1) + cart_lx(LC, ic)) * (LD + 1) +
                               cart_lx(LD, id);
                const int oy = ((cart_ly(LA, ia) * (LB + 1) + cart_ly(LB, ib)) * (LC + 1) + cart_ly(LC, ic)) * (LD + 1) +
                               cart_ly(LD, id);
                const int oz = ((cart_lz(LA, ia) * (LB + 1) + cart_lz(LB, ib)) * (LC + 1) + cart_lz(LC, ic)) * (LD + 1) +
                               cart_lz(LD, id);
                acc[ab * NCD + cd] = fmaf(gx[ox] * gy[oy], gz[oz], acc[ab * NCD + cd]);
            }
    }
}

// The same for the Obara--Saika classes: F_m(T) and the vertical
// recurrence in single precision, accumulated into the contracted [e0|f0].
template <int LA, int LB, int LC, int LD>
__device__ __forceinline__ void os_prim_quartet_f32(const QuartetGeomF &g, const float *P, const float *Q, float *v)
{
    constexpr int LT = LA + LB + LC + LD;
    const float zeta = P[0], eta = Q[0];
    const float PQ[3] = {P[2] - Q[2], P[3] - Q[3], P[4] - Q[4]};
    const float rs = rsqrtf(zeta + eta), izpe = rs * rs;
    const float T = zeta * eta * izpe * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
    const float pre = P[5] * Q[5] * rs;
    float F[LT + 1];
    boys_os_f32<LT>(T, F);
#pragma unroll
    for (int m = 0; m <= LT; ++m) F[m] *= pre;
    OsGeom<float> o;
    const float rz = eta * izpe, re = zeta * izpe;
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        o.PA[x] = P[2 + x] - g.A[x];
        o.QC[x] = Q[2 + x] - g.C[x];
        o.WP[x] = -rz * PQ[x];
        o.WQ[x] = re * PQ[x];
    }
    o.rz = rz;
    o.re = re;
    o.oo2z = 0.5f * P[1];
    o.oo2e = 0.5f * Q[1];
    o.oo2ze = 0.5f * izpe;
    OsClass<LA, LB, LC, LD>::template vrr<float>(o, F, v);
}

template <int LA, int LB, int LC, int LD, typename R, class Epi>
__global__ void __launch_bounds__(128, thread_min_blocks(ncart(LA) * ncart(LB) * ncart(LC) * ncart(LD)))
eri_thread_kernel(const int4 *__restrict__ list, int nq,
                                                         const PairInfo *__restrict__ pairs,
                                                         const PrimPair *__restrict__ prims, Epi epi)
{
    constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    constexpr int NAB = NA * NB, NCD = NC * ND;
    constexpr int NR = (LA + LB + LC + LD) / 2 + 1;
    constexpr int G2D = (LA + 1) * (LB + 1) * (LC + 1) * (LD + 1);
    // whole warps step through the list together (the J/K epilogue reduces
    // over the lanes); a lane past the end repeats the last item with no
    // primitive quartets
    const int lane = threadIdx.x & 31;
    for (int base = blockIdx.x * blockDim.x + threadIdx.x - lane; base < nq; base += gridDim.x * blockDim.x) {
        const int qi = base + lane;
        const bool live = qi < nq;
        int4 e = list[live ? qi : nq - 1];   // bra pair, ket pair, first primitive quartet, count
        if (!live) e.w = 0;
        const PairInfo &pb = pairs[e.x];
        const PairInfo &pk = pairs[e.y];
        // screened items (masked molecules, small density bounds) carry no
        // primitive quartets; a warp with none left skips the item altogether
        const bool skip = live && epi.screened(pb, pk, e.x, e.y);
        if (__all_sync(0xffffffffu, skip || !live)) continue;
        if (skip) e.w = 0;
        const double Ax = pb.A[0], Ay = pb.A[1], Az = pb.A[2];
        const double Cx = pk.A[0], Cy = pk.A[1], Cz = pk.A[2];
        const double ABx = pb.AB[0], ABy = pb.AB[1], ABz = pb.AB[2];
        const double CDx = pk.AB[0], CDy = pk.AB[1], CDz = pk.AB[2];
        R acc[NAB * NCD];
#pragma unroll
        for (int c = 0; c < NAB * NCD; ++c) acc[c] = (R)0;
        // primitive quartet g of the item = (bra primitive g % npb, ket
        // primitive g / npb): the bra index runs fastest, so the lanes of a
        // warp (which share the bra pair) step through the same bra
        // primitives and each lane fetches its own ket primitive pair only
        // once per npb steps
        const int npb = pb.nprim;
        const PrimPair *pbp = prims + pb.prim_off, *pkp = prims + pk.prim_off;
        int ik = e.z / npb, ib = e.z - (e.z / npb) * npb;
        if constexpr (std::is_same_v<R, float>) {
            // FP32 list of the mixed mode: single-precision primitive data
            QuartetGeomF gf;
#pragma unroll
            for (int x = 0; x < 3; ++x) {
                gf.A[x] = (float)pb.A[x];
                gf.C[x] = (float)pk.A[x];
                gf.AB[x] = (float)pb.AB[x];
                gf.CD[x] = (float)pk.AB[x];
            }
            float Pn[8], Q[8];
            ld8f(pbp[ib].f, Pn);
            ld8f(pkp[ik].f, Q);
            using OS = OsClass<LA, LB, LC, LD>;
            float v[OS::NV];
#pragma unroll
            for (int c = 0; c < OS::NV; ++c) v[c] = 0.0f;
            for (int t = 0; t < e.w; ++t) {
                float P[8];
#pragma unroll
                for (int c = 0; c < 8; ++c) P[c] = Pn[c];
                int ib2 = ib + 1, ik2 = ik;
                if (ib2 == npb) {
                    ib2 = 0;
                    ++ik2;
                }
                if (t + 1 < e.w) ld8f(pbp[ib2].f, Pn);
                float Qn[8];
                if (ik2 != ik && t + 1 < e.w) ld8f(pkp[ik2].f, Qn);
                if constexpr (OS::kOn)
                    os_prim_quartet_f32<LA, LB, LC, LD>(gf, P, Q, v);
                else
                    add_prim_quartet_f32<LA, LB, LC, LD>(gf, P, Q, reinterpret_cast<float *>(acc));
                if (ik2 != ik && t + 1 < e.w) {
#pragma unroll
                    for (int c = 0; c < 8; ++c) Q[c] = Qn[c];
                }
                ib = ib2;
                ik = ik2;
            }
            if constexpr (OS::kOn) OS::template hrr<float>(gf.AB, gf.CD, v, reinterpret_cast<float *>(acc));
            const QCtx q = make_qctx(pb, pk, e.x, e.y);
            epi.template thread_quartet<LA, LB, LC, LD, R>(q, acc, lane, live);
            continue;
        }
        PrimJK Pn = load_prim_jk(pbp + ib);
        PrimJK Q = load_prim_jk(pkp + ik);
        if constexpr (OsClass<LA, LB, LC, LD>::kOn) {
            // Obara--Saika per primitive quartet, Head-Gordon--Pople transfer
            // once per item on the contracted [e0|f0]
            using OS = OsClass<LA, LB, LC, LD>;
            constexpr int LT = LA + LB + LC + LD;
            R v[OS::NV];
#pragma unroll
            for (int c = 0; c < OS::NV; ++c) v[c] = (R)0;
            for (int t = 0; t < e.w; ++t) {
                const PrimJK P = Pn;
                int ib2 = ib + 1, ik2 = ik;
                if (ib2 == npb) {
                    ib2 = 0;
                    ++ik2;
                }
                if (t + 1 < e.w) Pn = load_prim_jk(pbp + ib2);
                // the next ket primitive pair, fetched a step ahead
                PrimJK Qn = Q;
                if (ik2 != ik && t + 1 < e.w) Qn = load_prim_jk(pkp + ik2);
                const double zeta = P.zeta, eta = Q.zeta;
                const double PQx = P.P[0] - Q.P[0], PQy = P.P[1] - Q.P[1], PQz = P.P[2] - Q.P[2];
                const double rs = rsqrt_nr_unchecked(zeta + eta);   // exponent sums: 1e-36 < x < 1e36
                const double izpe = rs * rs;
                const double T = zeta * eta * izpe * (PQx * PQx + PQy * PQy + PQz * PQz);
                const double pre = P.K * Q.K * rs;
                double F[LT + 1];
                boys_os<LT>(T, F);
                R Fs[LT + 1];
#pragma unroll
                for (int m = 0; m <= LT; ++m) Fs[m] = (R)(F[m] * pre);
                OsGeom<R> g;
                const double rz = eta * izpe, re = zeta * izpe;
                g.PA[0] = P.P[0] - Ax;
                g.PA[1] = P.P[1] - Ay;
                g.PA[2] = P.P[2] - Az;
                g.QC[0] = Q.P[0] - Cx;
                g.QC[1] = Q.P[1] - Cy;
                g.QC[2] = Q.P[2] - Cz;
                g.WP[0] = -rz * PQx;
                g.WP[1] = -rz * PQy;
                g.WP[2] = -rz * PQz;
                g.WQ[0] = re * PQx;
                g.WQ[1] = re * PQy;
                g.WQ[2] = re * PQz;
                g.rz = rz;
                g.re = re;
                g.oo2z = 0.5 * P.izeta;
                g.oo2e = 0.5 * Q.izeta;
                g.oo2ze = 0.5 * izpe;
                OS::template vrr<R>(g, Fs, v);
                Q = Qn;
                ib = ib2;
                ik = ik2;
            }
            const R AB[3] = {(R)ABx, (R)ABy, (R)ABz}, CD[3] = {(R)CDx, (R)CDy, (R)CDz};
            OS::template hrr<R>(AB, CD, v, acc);
            const QCtx q = make_qctx(pb, pk, e.x, e.y);
            epi.template thread_quartet<LA, LB, LC, LD, R>(q, acc, lane, live);
            continue;
        }
        for (int t = 0; t < e.w; ++t) {
            const PrimJK P = Pn;
            // the next bra primitive pair is fetched while this one computes
            int ib2 = ib + 1, ik2 = ik;
            if (ib2 == npb) {
                ib2 = 0;
                ++ik2;
            }
            if (t + 1 < e.w) Pn = load_prim_jk(pbp + ib2);
            const double zeta = P.zeta, eta = Q.zeta;
            const double PQx = P.P[0] - Q.P[0], PQy = P.P[1] - Q.P[1], PQz = P.P[2] - Q.P[2];
            const double rs = rsqrt_nr(zeta + eta);
            const double izpe = rs * rs;
            const double T = zeta * eta * izpe * (PQx * PQx + PQy * PQy + PQz * PQz);
            const double pre = P.K * Q.K * rs;
            double uu[NR], ww[NR];
            rys_roots_fast<NR>(T, uu, ww);
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                const RysCoef k = rys_coef(uu[r], zeta, eta, P.izeta, Q.izeta, izpe);
                R gx[G2D], gy[G2D], gz[G2D];
                rys2d_c<LA, LB, LC, LD, R>(k, P.P[0] - Ax, Q.P[0] - Cx, PQx, ABx, CDx, ww[r] * pre, gx);
                rys2d_c<LA, LB, LC, LD, R>(k, P.P[1] - Ay, Q.P[1] - Cy, PQy, ABy, CDy, 1.0, gy);
                rys2d_c<LA, LB, LC, LD, R>(k, P.P[2] - Az, Q.P[2] - Cz, PQz, ABz, CDz, 1.0, gz);
#pragma unroll
                for (int ab = 0; ab < NAB; ++ab)
#pragma unroll
                    for (int cd = 0; cd < NCD; ++cd) {
                        const int ia = ab / NB, ib3 = ab % NB, ic = cd / ND, id = cd % ND;
                        const int ox = ((cart_lx(LA, ia) * (LB + 1) + cart_lx(LB, ib3)) * (LC + 1) + cart_lx(LC, ic)) *
                                           (LD + 1) + cart_lx(LD, id);
                        const int oy = ((cart_ly(LA, ia) * (LB + 1) + cart_ly(LB, ib3)) * (LC + 1) + cart_ly(LC, ic)) *
                                           (LD + 1) + cart_ly(LD, id);
                        const int oz = ((cart_lz(LA, ia) * (LB + 1) + cart_lz(LB, ib3)) * (LC + 1) + cart_lz(LC, ic)) *
                                           (LD + 1) + cart_lz(LD, id);
                        acc[ab * NCD + cd] += gx[ox] * gy[oy] * gz[oz];
                    }
            }
            if (ik2 != ik && t + 1 < e.w) Q = load_prim_jk(pkp + ik2);
            ib = ib2;
            ik = ik2;
        }
        const QCtx q = make_qctx(pb, pk, e.x, e.y);
        epi.template thread_quartet<LA, LB, LC, LD, R>(q, acc, lane, live);
    }
}

// ----------------------------------------------------------- block mode --
constexpr int kBlockThreads = 256;

// Shared-memory budget of the 2-D integrals of one pass of a block: PB
// primitive quartets per slot go through the roots, 2-D and assembly phases
// together (two barriers per pass), as many as fit in the budget (at most 4).
constexpr size_t kBlockPassBytes = 64 * 1024;

template <int LA, int LB, int LC, int LD, typename R, class Epi>
struct BlockLayout {
    static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    static constexpr int NAB = NA * NB, NCD = NC * ND;
    static constexpr int NR = (LA + LB + LC + LD) / 2 + 1;
    static constexpr int G2D = (LA + 1) * (LB + 1) * (LC + 1) * (LD + 1);
    static constexpr int NSQ = kBlockThreads / NAB;
    static constexpr size_t pq_bytes = (size_t)NSQ * 3 * NR * G2D * sizeof(R);   // one primitive quartet per slot
    static constexpr int PB = pq_bytes * 4 <= kBlockPassBytes ? 4
                              : pq_bytes * 3 <= kBlockPassBytes ? 3
                              : pq_bytes * 2 <= kBlockPassBytes ? 2 : 1;
    static constexpr size_t g_bytes = (PB * pq_bytes + 15) / 16 * 16;
    // the integral tile of a tiled epilogue reuses the 2-D integral buffer
    static constexpr size_t tile_bytes = Epi::kTile ? (size_t)NSQ * NAB * (NCD + 1) * sizeof(double) : 0;
    static constexpr size_t bytes = g_bytes > tile_bytes ? g_bytes : tile_bytes;
};

struct SlotData {
    QCtx q;
    int npk, pp0, npp, pb_off, pk_off;
    double A[3], AB[3], C[3], CD[3];
};
struct SlotPrim {
    double zeta, eta, PA[3], QC[3], PQ[3];
};

// (the classes with at most six ket components fit three blocks per SM)
template <int LA, int LB, int LC, int LD, typename R, class Epi>
__global__ void __launch_bounds__(kBlockThreads, ncart(LC) * ncart(LD) <= 6 ? 3 : 0) eri_block_kernel(const int4 *__restrict__ list, int nq,
                                                                  const PairInfo *__restrict__ pairs,
                                                                  const PrimPair *__restrict__ prims, Epi epi)
{
    using Lay = BlockLayout<LA, LB, LC, LD, R, Epi>;
    constexpr int NB = Lay::NB, NC = Lay::NC, ND = Lay::ND, NAB = Lay::NAB, NCD = Lay::NCD;
    constexpr int NR = Lay::NR, G2D = Lay::G2D, NSQ = Lay::NSQ, PB = Lay::PB;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R *sg = reinterpret_cast<R *>(smem_raw);
    __shared__ SlotData sd[NSQ];
    __shared__ SlotPrim sp[PB][NSQ];
    __shared__ double su[PB][NSQ][NR], sw[PB][NSQ][NR];
    __shared__ int s_maxpp;

    const int tid = threadIdx.x;
    const int slot = tid / NAB, ab = tid - slot * NAB;
    const bool active = slot < NSQ;
    const int ia = active ? ab / NB : 0, ib = active ? ab % NB : 0;
    // offsets of this thread's bra component pair inside one (slot, axis, root) 2-D block
    const int ox = (cart_l(LA, ia, 0) * (LB + 1) + cart_l(LB, ib, 0)) * (LC + 1) * (LD + 1);
    const int oy = (cart_l(LA, ia, 1) * (LB + 1) + cart_l(LB, ib, 1)) * (LC + 1) * (LD + 1);
    const int oz = (cart_l(LA, ia, 2) * (LB + 1) + cart_l(LB, ib, 2)) * (LC + 1) * (LD + 1);

    for (int base = blockIdx.x * NSQ; base < nq; base += gridDim.x * NSQ) {
        if (tid == 0) s_maxpp = 0;
        __syncthreads();
        if (tid < NSQ) {
            SlotData &s = sd[tid];
            const int qi = base + tid;
            bool take = qi < nq;
            if (take) {
                const int4 t = list[qi];
                take = !epi.screened(pairs[t.x], pairs[t.y], t.x, t.y);
            }
            if (take) {
                const int4 e = list[qi];
                const PairInfo &pb = pairs[e.x];
                const PairInfo &pk = pairs[e.y];
                s.q = make_qctx(pb, pk, e.x, e.y);
                s.npk = pk.nprim;
                s.pp0 = e.z;
                s.npp = e.w;
                s.pb_off = pb.prim_off;
                s.pk_off = pk.prim_off;
                for (int x = 0; x < 3; ++x) {
                    s.A[x] = pb.A[x];
                    s.AB[x] = pb.AB[x];
                    s.C[x] = pk.A[x];
                    s.CD[x] = pk.AB[x];
                }
                atomicMax(&s_maxpp, s.npp);
            } else {
                s.q.bra = -1;
                s.npk = 1;
                s.pp0 = s.npp = 0;
                s.pb_off = s.pk_off = 0;
                for (int x = 0; x < 3; ++x) s.A[x] = s.AB[x] = s.C[x] = s.CD[x] = 0.0;
            }
        }
        __syncthreads();
        const int maxpp = s_maxpp;

        R acc[NCD];
#pragma unroll
        for (int c = 0; c < NCD; ++c) acc[c] = (R)0;

        for (int pp0 = 0; pp0 < maxpp; pp0 += PB) {
            // this pass: primitive quartets pp0 .. pp0 + nb - 1 of every slot
            const int nb = maxpp - pp0 < PB ? maxpp - pp0 : PB;
            // roots and weights (with the primitive-quartet prefactor)
            for (int t = tid; t < nb * NSQ * NR; t += kBlockThreads) {
                const int b = t / (NSQ * NR), rem = t - b * (NSQ * NR), s = rem / NR, r = rem - s * NR;
                const int pp = pp0 + b;
                const SlotData &S = sd[s];
                if (pp < S.npp) {
                    const int g = S.pp0 + pp;
                    const int jb = g / S.npk, jk = g - jb * S.npk;
                    const PrimPair P = prims[S.pb_off + jb];
                    const PrimPair Q = prims[S.pk_off + jk];
                    const double zpe = P.zeta + Q.zeta;
                    const double PQx = P.P[0] - Q.P[0], PQy = P.P[1] - Q.P[1], PQz = P.P[2] - Q.P[2];
                    const double T = P.zeta * Q.zeta / zpe * (PQx * PQx + PQy * PQy + PQz * PQz);
                    double u, w;
                    if constexpr (NR == 1) {
                        double uu[1], ww[1];
                        rys_roots<1>(T, uu, ww);
                        u = uu[0];
                        w = ww[0];
                    } else {
                        rys_root(NR, r, T, u, w);
                    }
                    su[b][s][r] = u;
                    sw[b][s][r] = w * P.K * Q.K * rsqrt(zpe);
                    if (r == 0) {
                        SlotPrim &p = sp[b][s];
                        p.zeta = P.zeta;
                        p.eta = Q.zeta;
                        p.PQ[0] = PQx;
                        p.PQ[1] = PQy;
                        p.PQ[2] = PQz;
                        for (int x = 0; x < 3; ++x) {
                            p.PA[x] = P.P[x] - S.A[x];
                            p.QC[x] = Q.P[x] - S.C[x];
                        }
                    }
                } else {
                    su[b][s][r] = 0.0;
                    sw[b][s][r] = 0.0;
                    if (r == 0) {
                        SlotPrim &p = sp[b][s];
                        p.zeta = p.eta = 1.0;
                        for (int x = 0; x < 3; ++x) p.PA[x] = p.QC[x] = p.PQ[x] = 0.0;
                    }
                }
            }
            __syncthreads();
            // 2-D integrals, one (pass quartet, slot, root, axis) per task; weight on x
            for (int t = tid; t < nb * NSQ * NR * 3; t += kBlockThreads) {
                const int b = t / (NSQ * NR * 3), rb = t - b * (NSQ * NR * 3);
                const int s = rb / (NR * 3), rem = rb - s * NR * 3, r = rem / 3, x = rem - r * 3;
                const SlotPrim &p = sp[b][s];
                rys2d<LA, LB, LC, LD, R>(su[b][s][r], p.zeta, p.eta, p.PA[x], p.QC[x], p.PQ[x], sd[s].AB[x],
                                         sd[s].CD[x], x == 0 ? sw[b][s][r] : 1.0,
                                         sg + ((size_t)((b * NSQ + s) * 3 + x) * NR + r) * G2D);
            }
            __syncthreads();
            // assembly: this thread's bra pair (ia, ib) times every ket pair
            if (active) {
                for (int b = 0; b < nb; ++b) {
                    const R *gx = sg + (size_t)((b * NSQ + slot) * 3 + 0) * NR * G2D + ox;
                    const R *gy = sg + (size_t)((b * NSQ + slot) * 3 + 1) * NR * G2D + oy;
                    const R *gz = sg + (size_t)((b * NSQ + slot) * 3 + 2) * NR * G2D + oz;
#pragma unroll
                    for (int r = 0; r < NR; ++r)
#pragma unroll
                        for (int ic = 0; ic < NC; ++ic)
#pragma unroll
                            for (int id = 0; id < ND; ++id) {
                                const int cx = cart_lx(LC, ic) * (LD + 1) + cart_lx(LD, id);
                                const int cy = cart_ly(LC, ic) * (LD + 1) + cart_ly(LD, id);
                                const int cz = cart_lz(LC, ic) * (LD + 1) + cart_lz(LD, id);
                                acc[ic * ND + id] += gx[r * G2D + cx] * gy[r * G2D + cy] * gz[r * G2D + cz];
                            }
                }
            }
        }

        if constexpr (Epi::kTile) {
            constexpr int ST = NCD + 1;
            double *V = reinterpret_cast<double *>(smem_raw) + (size_t)slot * NAB * ST;
            __syncthreads();   // the tile overwrites the 2-D integrals
            if (active && sd[slot].q.bra >= 0) epi.template tile_store<LA, LB, LC, LD, R>(sd[slot].q, ia, ib, acc, V);
            __syncthreads();
            if (active && sd[slot].q.bra >= 0) epi.template tile_reduce<LA, LB, LC, LD>(sd[slot].q, V, ab, NAB);
        } else {
            if (active && sd[slot].q.bra >= 0) epi.template block_ab<LA, LB, LC, LD, R>(sd[slot].q, ia, ib, acc);
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------- dispatch --
template <int LA, int LB, int LC, int LD>
struct ClassTag {};

__host__ __device__ constexpr int pc_la(int c) { return c == 0 ? 0 : (c <= 2 ? 1 : 2); }
__host__ __device__ constexpr int pc_lb(int c) { return c == 0 ? 0 : (c == 1 ? 0 : (c == 2 ? 1 : c - 3)); }

template <int LA, int LB, int LC, int LD, typename R, class Epi>
inline cudaError_t launch_eri_class(const int4 *list, int nq, const PairInfo *pairs, const PrimPair *prims,
                                    const Epi &epi, cudaStream_t st, int nsm)
{
    if (nq <= 0) return cudaSuccess;
    constexpr int NAB = ncart(LA) * ncart(LB), NCD = ncart(LC) * ncart(LD);
    // thread mode while the contracted components fit in registers
    constexpr int kThreadMax = 81;
    if constexpr (NAB * NCD <= kThreadMax) {
        int grid = (nq + 127) / 128;
        if (grid > nsm * 32) grid = nsm * 32;
        eri_thread_kernel<LA, LB, LC, LD, R, Epi><<<grid, 128, 0, st>>>(list, nq, pairs, prims, epi);
    } else {
        using Lay = BlockLayout<LA, LB, LC, LD, R, Epi>;
        auto kern = eri_block_kernel<LA, LB, LC, LD, R, Epi>;
        // the attribute is per device: set once per instantiation and device
        static std::atomic<unsigned long long> attr_set{0};
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
        if (!bit || !(attr_set.load() & bit)) {
            e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Lay::bytes);
            if (e != cudaSuccess) return e;
            attr_set.fetch_or(bit);
        }
        int grid = (nq + Lay::NSQ - 1) / Lay::NSQ;
        if (grid > nsm * 8) grid = nsm * 8;
        kern<<<grid, kBlockThreads, Lay::bytes, st>>>(list, nq, pairs, prims, epi);
    }
    return cudaGetLastError();
}

// Run class `qc` (0..20): bra pair class cb >= ket pair class ck.
template <typename R, class Epi>
inline cudaError_t launch_eri(int qc, const int4 *list, int nq, const PairInfo *pairs, const PrimPair *prims,
                              const Epi &epi, cudaStream_t st, int nsm)
{
#define PQB_CASE(CB, CK)                                                                                       \
    case CB *(CB + 1) / 2 + CK:                                                                               \
        return launch_eri_class<pc_la(CB), pc_lb(CB), pc_la(CK), pc_lb(CK), R, Epi>(list, nq, pairs, prims, epi, \
                                                                                    st, nsm);
    switch (qc) {
        PQB_CASE(0, 0)
        PQB_CASE(1, 0) PQB_CASE(1, 1)
        PQB_CASE(2, 0) PQB_CASE(2, 1) PQB_CASE(2, 2)
        PQB_CASE(3, 0) PQB_CASE(3, 1) PQB_CASE(3, 2) PQB_CASE(3, 3)
        PQB_CASE(4, 0) PQB_CASE(4, 1) PQB_CASE(4, 2) PQB_CASE(4, 3) PQB_CASE(4, 4)
        PQB_CASE(5, 0) PQB_CASE(5, 1) PQB_CASE(5, 2) PQB_CASE(5, 3) PQB_CASE(5, 4) PQB_CASE(5, 5)
    }
#undef PQB_CASE
    return cudaErrorInvalidValue;
}

}  // namespace pqb
