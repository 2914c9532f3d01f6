// Shell-quartet ERI engine: one kernel template per angular-momentum class
// (LA LB | LC LD), fed a class-sorted list of (bra pair, ket pair) quartets.
//
// The integral is the Rys quadrature of the reference's Src/crys.c:56-97
// (sum over roots of Ix*Iy*Iz*w, ABD eqs 5, 9), but organised per SHELL
// quartet: roots and 2-D integrals are computed once per primitive quartet
// and shared by every cartesian component, instead of once per component as
// crys.contr_coulomb does (Src/crys.c:34-54).
//
// Two execution modes:
//  * thread mode (NAB*NCD <= 54 in FP64, <= 81 in FP32): one thread per quartet,
//    2-D integrals and all contracted components live in registers.
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
//   thread_quartet<LA,LB,LC,LD>(q, acc[NAB*NCD])   whole quartet, thread mode
//   block_ab<LA,LB,LC,LD>(q, ia, ib, acc[NCD], scr) one bra component pair,
//                                                    block mode (scr: per-slot
//                                                    shared scratch)
//   block_flush<LA,LB,LC,LD>(q, scr, t, nt)          after a block barrier
//   kScratch<LA,LB,LC,LD>                            doubles of scr per slot

__device__ __forceinline__ bool skip_bra(const QCtx &q, int fi, int fj) { return q.sa == q.sb && fi < fj; }

// Packed canonical integrals at ijkl2intindex (Src/cints.c:413-425), 64-bit.
struct EpiPacked {
    double *out;
    const double *fscale;
    template <int LA, int LB, int LC, int LD>
    static constexpr int kScratch = 0;
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
    __device__ __forceinline__ void thread_quartet(const QCtx &q, const R *acc) const
    {
        constexpr int NB = ncart(LB), NCD = ncart(LC) * ncart(LD);
#pragma unroll
        for (int ab = 0; ab < ncart(LA) * NB; ++ab) this->ab<LC, LD, R>(q, ab / NB, ab % NB, acc + ab * NCD);
    }
    template <int LA, int LB, int LC, int LD, typename R>
    __device__ __forceinline__ void block_ab(const QCtx &q, int ia, int ib, const R *acc, double *) const
    {
        ab<LC, LD, R>(q, ia, ib, acc);
    }
    template <int LA, int LB, int LC, int LD>
    __device__ __forceinline__ void block_flush(const QCtx &, double *, int, int) const {}
};

// Direct J/K digestion of unique quartets with 8-fold degeneracy weights:
//   Jacc[i,j] += 2 v' D_kl,  Jacc[k,l] += 2 v' D_ij,
//   Kacc[i,k] += v' D_jl, Kacc[i,l] += v' D_jk, Kacc[j,k] += v' D_il, Kacc[j,l] += v' D_ik,
// v' = v * (1/2 if i==j) (1/2 if k==l) (1/2 if ij==kl); then J = Jacc + Jacc^T,
// K = Kacc + Kacc^T reproduce J_ij = sum_kl (ij|kl) D_kl and
// K_ij = sum_kl (ik|jl) D_kl of PyQuante/Ints.py:195-223 for symmetric D.
// Contributions are first summed per quartet into its six J/K blocks
// (ab, cd, ac, ad, bc, bd) and then added to global memory once per block
// element, so a quartet costs NA NB + NC ND + (NA+NB)(NC+ND) atomics.
struct EpiJK {
    const double *D;
    double *Jacc, *Kacc;
    const double *fscale;
    template <int LA, int LB, int LC, int LD>
    static constexpr int kScratch = ncart(LA) * ncart(LB) + ncart(LC) * ncart(LD) +
                                    (ncart(LA) + ncart(LB)) * (ncart(LC) + ncart(LD));

    // digest one bra component pair: returns 2*sum_kl v' D_kl (the Jacc[i,j]
    // term) and adds the other five block contributions through the sinks
    template <int LC, int LD, typename R, class Sink>
    __device__ __forceinline__ double ab(const QCtx &q, int ia, int ib, const R *acc, Sink &&sink) const
    {
        constexpr int NC = ncart(LC), ND = ncart(LD);
        const int fi = q.fa + ia, fj = q.fb + ib;
        if (skip_bra(q, fi, fj)) return 0.0;
        const int64_t IJ = fpair(fi, fj);
        const double sij = fscale[fi] * fscale[fj] * (fi == fj ? 0.5 : 1.0);
        const double *Db = D + q.bo;
        const int nm = q.nm;
        const double Dij = __ldg(Db + (int64_t)fi * nm + fj);
        const double *Di = Db + (int64_t)fi * nm, *Dj = Db + (int64_t)fj * nm;
        double jij = 0.0;
#pragma unroll
        for (int ic = 0; ic < NC; ++ic) {
            double kik = 0.0, kjk = 0.0;
#pragma unroll
            for (int id = 0; id < ND; ++id) {
                const int fk = q.fc + ic, fl = q.fd + id;
                if (q.sc == q.sd && fk < fl) continue;
                const int64_t KL = fpair(fk, fl);
                if (q.bra == q.ket && IJ < KL) continue;
                const double v = (double)acc[ic * ND + id] * sij * fscale[fk] * fscale[fl] *
                                 (fk == fl ? 0.5 : 1.0) * (IJ == KL ? 0.5 : 1.0);
                jij += v * __ldg(Db + (int64_t)fk * nm + fl);
                sink.jcd(ic * ND + id, 2.0 * v * Dij);
                kik += v * __ldg(Dj + fl);
                kjk += v * __ldg(Di + fl);
                sink.kad(ia, id, v * __ldg(Dj + fk));
                sink.kbd(ib, id, v * __ldg(Di + fk));
            }
            sink.kac(ia, ic, kik);
            sink.kbc(ib, ic, kjk);
        }
        return 2.0 * jij;
    }

    // thread mode: block sums in registers, then one atomic per element
    template <int LA, int LB, int LC, int LD, typename R>
    __device__ __forceinline__ void thread_quartet(const QCtx &q, const R *acc) const
    {
        constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD), NCD = NC * ND;
        struct Regs {
            double jcd_[NCD], kac_[NC], kad_[ND], kbc_[NB][NC], kbd_[NB][ND];
            __device__ void jcd(int c, double v) { jcd_[c] += v; }
            __device__ void kac(int, int c, double v) { kac_[c] += v; }
            __device__ void kad(int, int d, double v) { kad_[d] += v; }
            __device__ void kbc(int b, int c, double v) { kbc_[b][c] += v; }
            __device__ void kbd(int b, int d, double v) { kbd_[b][d] += v; }
        } r;
#pragma unroll
        for (int c = 0; c < NCD; ++c) r.jcd_[c] = 0.0;
#pragma unroll
        for (int b = 0; b < NB; ++b) {
#pragma unroll
            for (int c = 0; c < NC; ++c) r.kbc_[b][c] = 0.0;
#pragma unroll
            for (int d = 0; d < ND; ++d) r.kbd_[b][d] = 0.0;
        }
#pragma unroll
        for (int ia = 0; ia < NA; ++ia) {
#pragma unroll
            for (int c = 0; c < NC; ++c) r.kac_[c] = 0.0;
#pragma unroll
            for (int d = 0; d < ND; ++d) r.kad_[d] = 0.0;
#pragma unroll
            for (int ib = 0; ib < NB; ++ib) {
                const double jij = ab<LC, LD, R>(q, ia, ib, acc + (ia * NB + ib) * NCD, r);
                if (jij != 0.0) atomicAdd(Jacc + q.bo + (int64_t)(q.fa + ia) * q.nm + q.fb + ib, jij);
            }
#pragma unroll
            for (int c = 0; c < NC; ++c)
                if (r.kac_[c] != 0.0) atomicAdd(Kacc + q.bo + (int64_t)(q.fa + ia) * q.nm + q.fc + c, r.kac_[c]);
#pragma unroll
            for (int d = 0; d < ND; ++d)
                if (r.kad_[d] != 0.0) atomicAdd(Kacc + q.bo + (int64_t)(q.fa + ia) * q.nm + q.fd + d, r.kad_[d]);
        }
#pragma unroll
        for (int b = 0; b < NB; ++b) {
#pragma unroll
            for (int c = 0; c < NC; ++c)
                if (r.kbc_[b][c] != 0.0) atomicAdd(Kacc + q.bo + (int64_t)(q.fb + b) * q.nm + q.fc + c, r.kbc_[b][c]);
#pragma unroll
            for (int d = 0; d < ND; ++d)
                if (r.kbd_[b][d] != 0.0) atomicAdd(Kacc + q.bo + (int64_t)(q.fb + b) * q.nm + q.fd + d, r.kbd_[b][d]);
        }
#pragma unroll
        for (int c = 0; c < NCD; ++c)
            if (r.jcd_[c] != 0.0) atomicAdd(Jacc + q.bo + (int64_t)(q.fc + c / ND) * q.nm + q.fd + c % ND, r.jcd_[c]);
    }

    // block mode: scratch layout [jab NAB | jcd NCD | kac NA*NC | kad NA*ND | kbc NB*NC | kbd NB*ND]
    template <int LA, int LB, int LC, int LD, typename R>
    __device__ __forceinline__ void block_ab(const QCtx &q, int ia, int ib, const R *acc, double *scr) const
    {
        constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
        struct Smem {
            double *s;
            __device__ void jcd(int c, double v) { atomicAdd(s + NA * NB + c, v); }
            __device__ void kac(int a, int c, double v) { atomicAdd(s + NA * NB + NC * ND + a * NC + c, v); }
            __device__ void kad(int a, int d, double v) { atomicAdd(s + NA * NB + NC * ND + NA * NC + a * ND + d, v); }
            __device__ void kbc(int b, int c, double v)
            {
                atomicAdd(s + NA * NB + NC * ND + NA * NC + NA * ND + b * NC + c, v);
            }
            __device__ void kbd(int b, int d, double v)
            {
                atomicAdd(s + NA * NB + NC * ND + NA * NC + NA * ND + NB * NC + b * ND + d, v);
            }
        } sm{scr};
        scr[ia * NB + ib] = ab<LC, LD, R>(q, ia, ib, acc, sm);
    }
    template <int LA, int LB, int LC, int LD>
    __device__ __forceinline__ void block_flush(const QCtx &q, const double *scr, int t, int nt) const
    {
        constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
        constexpr int O1 = NA * NB, O2 = O1 + NC * ND, O3 = O2 + NA * NC, O4 = O3 + NA * ND, O5 = O4 + NB * NC,
                      O6 = O5 + NB * ND;
        for (int e = t; e < O6; e += nt) {
            const double v = scr[e];
            if (v == 0.0) continue;
            int row, col;
            double *M = Kacc;
            if (e < O1) { row = q.fa + e / NB; col = q.fb + e % NB; M = Jacc; }
            else if (e < O2) { row = q.fc + (e - O1) / ND; col = q.fd + (e - O1) % ND; M = Jacc; }
            else if (e < O3) { row = q.fa + (e - O2) / NC; col = q.fc + (e - O2) % NC; }
            else if (e < O4) { row = q.fa + (e - O3) / ND; col = q.fd + (e - O3) % ND; }
            else if (e < O5) { row = q.fb + (e - O4) / NC; col = q.fc + (e - O4) % NC; }
            else { row = q.fb + (e - O5) / ND; col = q.fd + (e - O5) % ND; }
            atomicAdd(M + q.bo + (int64_t)row * q.nm + col, v);
        }
    }
};

// Schwarz: Q2[pair] = max over components of |(ij|ij)| (diagonal quartets).
struct EpiSchwarz {
    unsigned long long *Q2bits;   // bit patterns of non-negative doubles
    const double *fscale;
    template <int LA, int LB, int LC, int LD>
    static constexpr int kScratch = 0;
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
    __device__ __forceinline__ void thread_quartet(const QCtx &q, const R *acc) const
    {
        constexpr int NB = ncart(LB), NCD = ncart(LC) * ncart(LD);
#pragma unroll
        for (int ab = 0; ab < ncart(LA) * NB; ++ab) this->ab<LC, LD, R>(q, ab / NB, ab % NB, acc + ab * NCD);
    }
    template <int LA, int LB, int LC, int LD, typename R>
    __device__ __forceinline__ void block_ab(const QCtx &q, int ia, int ib, const R *acc, double *) const
    {
        ab<LC, LD, R>(q, ia, ib, acc);
    }
    template <int LA, int LB, int LC, int LD>
    __device__ __forceinline__ void block_flush(const QCtx &, double *, int, int) const {}
};

// ---------------------------------------------------------- thread mode --
// Register cap per class (via the minimum resident blocks of 128 threads):
// small classes are latency bound, so they trade registers for occupancy.
__host__ __device__ constexpr int thread_min_blocks(int nabcd) { return nabcd == 1 ? 8 : (nabcd <= 9 ? 4 : 2); }

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
    for (int qi = blockIdx.x * blockDim.x + threadIdx.x; qi < nq; qi += gridDim.x * blockDim.x) {
        const int4 e = list[qi];   // bra pair, ket pair, first primitive quartet, count
        const PairInfo &pb = pairs[e.x];
        const PairInfo &pk = pairs[e.y];
        const double Ax = pb.A[0], Ay = pb.A[1], Az = pb.A[2];
        const double Cx = pk.A[0], Cy = pk.A[1], Cz = pk.A[2];
        const double ABx = pb.AB[0], ABy = pb.AB[1], ABz = pb.AB[2];
        const double CDx = pk.AB[0], CDy = pk.AB[1], CDz = pk.AB[2];
        R acc[NAB * NCD];
#pragma unroll
        for (int c = 0; c < NAB * NCD; ++c) acc[c] = (R)0;
        const int npk = pk.nprim;
        int ib = e.z / npk, ik = e.z - (e.z / npk) * npk;
        PrimPair P = prims[pb.prim_off + ib];
        for (int t = 0; t < e.w; ++t) {
            const PrimPair Q = prims[pk.prim_off + ik];
            const double zpe = P.zeta + Q.zeta;
            const double PQx = P.P[0] - Q.P[0], PQy = P.P[1] - Q.P[1], PQz = P.P[2] - Q.P[2];
            const double T = P.zeta * Q.zeta / zpe * (PQx * PQx + PQy * PQy + PQz * PQz);
            const double pre = P.K * Q.K * rsqrt(zpe);
            double uu[NR], ww[NR];
            rys_roots<NR>(T, uu, ww);
#pragma unroll
            for (int r = 0; r < NR; ++r) {
                const double u = uu[r], w = ww[r];
                R gx[G2D], gy[G2D], gz[G2D];
                rys2d<LA, LB, LC, LD, R>(u, P.zeta, Q.zeta, P.P[0] - Ax, Q.P[0] - Cx, PQx, ABx, CDx, w * pre, gx);
                rys2d<LA, LB, LC, LD, R>(u, P.zeta, Q.zeta, P.P[1] - Ay, Q.P[1] - Cy, PQy, ABy, CDy, 1.0, gy);
                rys2d<LA, LB, LC, LD, R>(u, P.zeta, Q.zeta, P.P[2] - Az, Q.P[2] - Cz, PQz, ABz, CDz, 1.0, gz);
#pragma unroll
                for (int ab = 0; ab < NAB; ++ab)
#pragma unroll
                    for (int cd = 0; cd < NCD; ++cd) {
                        const int ia = ab / NB, ib2 = ab % NB, ic = cd / ND, id = cd % ND;
                        const int ox = ((cart_lx(LA, ia) * (LB + 1) + cart_lx(LB, ib2)) * (LC + 1) + cart_lx(LC, ic)) *
                                           (LD + 1) + cart_lx(LD, id);
                        const int oy = ((cart_ly(LA, ia) * (LB + 1) + cart_ly(LB, ib2)) * (LC + 1) + cart_ly(LC, ic)) *
                                           (LD + 1) + cart_ly(LD, id);
                        const int oz = ((cart_lz(LA, ia) * (LB + 1) + cart_lz(LB, ib2)) * (LC + 1) + cart_lz(LC, ic)) *
                                           (LD + 1) + cart_lz(LD, id);
                        acc[ab * NCD + cd] += gx[ox] * gy[oy] * gz[oz];
                    }
            }
            if (++ik == npk) {
                ik = 0;
                ++ib;
                if (t + 1 < e.w) P = prims[pb.prim_off + ib];
            }
        }
        const QCtx q = make_qctx(pb, pk, e.x, e.y);
        epi.template thread_quartet<LA, LB, LC, LD, R>(q, acc);
    }
}

// ----------------------------------------------------------- block mode --
constexpr int kBlockThreads = 256;

template <int LA, int LB, int LC, int LD, typename R, class Epi>
struct BlockLayout {
    static constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    static constexpr int NAB = NA * NB, NCD = NC * ND;
    static constexpr int NR = (LA + LB + LC + LD) / 2 + 1;
    static constexpr int G2D = (LA + 1) * (LB + 1) * (LC + 1) * (LD + 1);
    static constexpr int NSQ = kBlockThreads / NAB;
    static constexpr int SCR = Epi::template kScratch<LA, LB, LC, LD>;
    static constexpr size_t g_bytes = ((size_t)NSQ * 3 * NR * G2D * sizeof(R) + 15) / 16 * 16;
    static constexpr size_t scr_bytes = (size_t)NSQ * SCR * sizeof(double);
    static constexpr size_t bytes = g_bytes + scr_bytes;
};

struct SlotData {
    QCtx q;
    int npk, pp0, npp, pb_off, pk_off;
    double A[3], AB[3], C[3], CD[3];
};
struct SlotPrim {
    double zeta, eta, PA[3], QC[3], PQ[3];
};

template <int LA, int LB, int LC, int LD, typename R, class Epi>
__global__ void __launch_bounds__(kBlockThreads) eri_block_kernel(const int4 *__restrict__ list, int nq,
                                                                  const PairInfo *__restrict__ pairs,
                                                                  const PrimPair *__restrict__ prims, Epi epi)
{
    using Lay = BlockLayout<LA, LB, LC, LD, R, Epi>;
    constexpr int NB = Lay::NB, NC = Lay::NC, ND = Lay::ND, NAB = Lay::NAB, NCD = Lay::NCD;
    constexpr int NR = Lay::NR, G2D = Lay::G2D, NSQ = Lay::NSQ, SCR = Lay::SCR;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R *sg = reinterpret_cast<R *>(smem_raw);
    double *sscr = reinterpret_cast<double *>(smem_raw + Lay::g_bytes);
    __shared__ SlotData sd[NSQ];
    __shared__ SlotPrim sp[NSQ];
    __shared__ double su[NSQ][NR], sw[NSQ][NR];
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
            if (qi < nq) {
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
        if constexpr (SCR > 0)
            for (int t = tid; t < NSQ * SCR; t += kBlockThreads) sscr[t] = 0.0;
        __syncthreads();
        const int maxpp = s_maxpp;

        R acc[NCD];
#pragma unroll
        for (int c = 0; c < NCD; ++c) acc[c] = (R)0;

        for (int pp = 0; pp < maxpp; ++pp) {
            // roots and weights (with the primitive-quartet prefactor)
            for (int t = tid; t < NSQ * NR; t += kBlockThreads) {
                const int s = t / NR, r = t - s * NR;
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
                    su[s][r] = u;
                    sw[s][r] = w * P.K * Q.K * rsqrt(zpe);
                    if (r == 0) {
                        SlotPrim &p = sp[s];
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
                    su[s][r] = 0.0;
                    sw[s][r] = 0.0;
                    if (r == 0) {
                        SlotPrim &p = sp[s];
                        p.zeta = p.eta = 1.0;
                        for (int x = 0; x < 3; ++x) p.PA[x] = p.QC[x] = p.PQ[x] = 0.0;
                    }
                }
            }
            __syncthreads();
            // 2-D integrals, one (slot, root, axis) per task; weight on x
            for (int t = tid; t < NSQ * NR * 3; t += kBlockThreads) {
                const int s = t / (NR * 3), rem = t - s * NR * 3, r = rem / 3, x = rem - r * 3;
                const SlotPrim &p = sp[s];
                rys2d<LA, LB, LC, LD, R>(su[s][r], p.zeta, p.eta, p.PA[x], p.QC[x], p.PQ[x], sd[s].AB[x], sd[s].CD[x],
                                         x == 0 ? sw[s][r] : 1.0, sg + ((size_t)(s * 3 + x) * NR + r) * G2D);
            }
            __syncthreads();
            // assembly: this thread's bra pair (ia, ib) times every ket pair
            if (active) {
                const R *gx = sg + (size_t)(slot * 3 + 0) * NR * G2D + ox;
                const R *gy = sg + (size_t)(slot * 3 + 1) * NR * G2D + oy;
                const R *gz = sg + (size_t)(slot * 3 + 2) * NR * G2D + oz;
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

        if (active && sd[slot].q.bra >= 0)
            epi.template block_ab<LA, LB, LC, LD, R>(sd[slot].q, ia, ib, acc, sscr + slot * SCR);
        if constexpr (SCR > 0) {
            __syncthreads();
            // flush: NAB threads per slot walk the slot's scratch
            if (active && sd[slot].q.bra >= 0)
                epi.template block_flush<LA, LB, LC, LD>(sd[slot].q, sscr + slot * SCR, ab, NAB);
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
        static bool attr_set = false;   // per instantiation
        if (!attr_set) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Lay::bytes);
            if (e != cudaSuccess) return e;
            attr_set = true;
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
