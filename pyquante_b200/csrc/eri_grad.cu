// Nuclear gradient of the two-electron energy, contracted on the fly:
//
//   dE2/dX = sum over unique (ij|kl) of  d(ij|kl)/dX * Gamma_ijkl,
//   Gamma_ijkl = 8 s (2 D_ij D_kl - (D_ik D_jl + D_il D_jk)/2),
//
// s the 8-fold degeneracy weight (1/2 per i==j, k==l, ij==kl), which is
// E2 = sum_ijkl (ij|kl)(2 D_ij D_kl - D_ik D_jl) of the RHF energy
// E = tr(D h) + tr(D F) (PyQuante/hartree_fock.py:33-38) differentiated; the
// reference forms it as trace2(D, der2JmK(...)) over stored derivative
// integrals (PyQuante/force.py:106-116,232-252,318-357).
//
// Derivative integrals come from the same Rys 2-D integrals with one more
// unit of momentum on the bra and ket centres A, B, C:
//   d/dA_x phi_a = 2 alpha_a phi_{a+1x} - a_x phi_{a-1x}
// (the raising/lowering relation of PyQuante/AnalyticDerivatives.py, applied
// to each primitive), and the fourth centre by translational invariance,
// dD = -(dA + dB + dC).  One thread per work item (quartet, primitive
// chunk); the component loops stay rolled (the derivative kernel favours
// compact code over peak speed); nine gradient components accumulate in
// registers and go to the four atoms with twelve atomics.
#include "eri_engine.cuh"
#include "eri_launch.h"

namespace pqb {

template <int LA, int LB, int LC, int LD, typename R>
__global__ void __launch_bounds__(128) eri_grad_kernel(const int4 *__restrict__ list, int nq,
                                                       const PairInfo *__restrict__ pairs,
                                                       const PrimPair *__restrict__ prims,
                                                       const double *__restrict__ D, const double *__restrict__ fscale,
                                                       const int *__restrict__ shell_atom, int n, double *grad)
{
    constexpr int NA = ncart(LA), NB = ncart(LB), NC = ncart(LC), ND = ncart(LD);
    constexpr int NAB = NA * NB, NCD = NC * ND;
    constexpr int NR = (LA + LB + LC + LD + 1) / 2 + 1;
    constexpr int EA = LA + 1, EB = LB + 1, EC = LC + 1, ED = LD;
    constexpr int G2 = (EA + 1) * (EB + 1) * (EC + 1) * (ED + 1);
    // component exponents packed per shell component: x | y << 4 | z << 8
    auto pk3 = [](int L, int i) { return cart_lx(L, i) | (cart_ly(L, i) << 4) | (cart_lz(L, i) << 8); };
    for (int qi = blockIdx.x * blockDim.x + threadIdx.x; qi < nq; qi += gridDim.x * blockDim.x) {
        const int4 e = list[qi];
        const PairInfo &pb = pairs[e.x];
        const PairInfo &pk = pairs[e.y];
        const QCtx q = make_qctx(pb, pk, e.x, e.y);
        // Gamma for every component of the quartet (0 for non-canonical ones)
        double gam[NAB * NCD];
#pragma unroll 1
        for (int ab = 0; ab < NAB; ++ab) {
            const int fi = q.fa + ab / NB, fj = q.fb + ab % NB;
            const int64_t IJ = fpair(fi, fj);
#pragma unroll 1
            for (int cd = 0; cd < NCD; ++cd) {
                const int fk = q.fc + cd / ND, fl = q.fd + cd % ND;
                const int64_t KL = fpair(fk, fl);
                double g = 0.0;
                if (!((q.sa == q.sb && fi < fj) || (q.sc == q.sd && fk < fl) || (q.bra == q.ket && IJ < KL))) {
                    const double s = 8.0 * (fi == fj ? 0.5 : 1.0) * (fk == fl ? 0.5 : 1.0) * (IJ == KL ? 0.5 : 1.0) *
                                     fscale[fi] * fscale[fj] * fscale[fk] * fscale[fl];
                    const double *Db = D + q.bo;
                    const int nm = q.nm;
                    const double dij = __ldg(Db + (int64_t)fi * nm + fj), dkl = __ldg(Db + (int64_t)fk * nm + fl);
                    const double dik = __ldg(Db + (int64_t)fi * nm + fk), djl = __ldg(Db + (int64_t)fj * nm + fl);
                    const double dil = __ldg(Db + (int64_t)fi * nm + fl), djk = __ldg(Db + (int64_t)fj * nm + fk);
                    g = s * (2.0 * dij * dkl - 0.5 * (dik * djl + dil * djk));
                }
                gam[ab * NCD + cd] = g;
            }
        }
        double gA[3] = {0, 0, 0}, gB[3] = {0, 0, 0}, gC[3] = {0, 0, 0};
        const int npk = pk.nprim;
        int ib = e.z / npk, ik = e.z - (e.z / npk) * npk;
#pragma unroll 1
        for (int t = 0; t < e.w; ++t) {
            const PrimPair P = prims[pb.prim_off + ib];
            const PrimPair Q = prims[pk.prim_off + ik];
            if (++ik == npk) {
                ik = 0;
                ++ib;
            }
            const R aa2 = (R)(2.0 * P.alpha_a), ab2 = (R)(2.0 * (P.zeta - P.alpha_a)), ac2 = (R)(2.0 * Q.alpha_a);
            const double zpe = P.zeta + Q.zeta;
            const double PQ[3] = {P.P[0] - Q.P[0], P.P[1] - Q.P[1], P.P[2] - Q.P[2]};
            const double T = P.zeta * Q.zeta / zpe * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
            const double pre = P.K * Q.K * rsqrt(zpe);
            double uu[NR], ww[NR];
            rys_roots<NR>(T, uu, ww);
#pragma unroll 1
            for (int r = 0; r < NR; ++r) {
                R g[3][G2];
#pragma unroll
                for (int x = 0; x < 3; ++x)
                    rys2d<EA, EB, EC, ED, R>(uu[r], P.zeta, Q.zeta, P.P[x] - pb.A[x], Q.P[x] - pk.A[x], PQ[x], pb.AB[x],
                                             pk.AB[x], x == 0 ? ww[r] * pre : 1.0, g[x]);
#pragma unroll 1
                for (int ab = 0; ab < NAB; ++ab) {
                    const int pa = pk3(LA, ab / NB), pbb = pk3(LB, ab % NB);
#pragma unroll 1
                    for (int cd = 0; cd < NCD; ++cd) {
                        const double gm = gam[ab * NCD + cd];
                        if (gm == 0.0) continue;
                        const int pc = pk3(LC, cd / ND), pd = pk3(LD, cd % ND);
                        R I[3], dA[3], dB[3], dC[3];
#pragma unroll
                        for (int x = 0; x < 3; ++x) {
                            const int a = (pa >> (4 * x)) & 15, b = (pbb >> (4 * x)) & 15, c = (pc >> (4 * x)) & 15,
                                      d = (pd >> (4 * x)) & 15;
                            const R *gx = g[x];
                            const int i0 = ((a * (EB + 1) + b) * (EC + 1) + c) * (ED + 1) + d;
                            constexpr int sA = (EB + 1) * (EC + 1) * (ED + 1), sB = (EC + 1) * (ED + 1), sC = ED + 1;
                            I[x] = gx[i0];
                            dA[x] = aa2 * gx[i0 + sA] - (a > 0 ? (R)a * gx[i0 - sA] : (R)0);
                            dB[x] = ab2 * gx[i0 + sB] - (b > 0 ? (R)b * gx[i0 - sB] : (R)0);
                            dC[x] = ac2 * gx[i0 + sC] - (c > 0 ? (R)c * gx[i0 - sC] : (R)0);
                        }
                        gA[0] += gm * (double)(dA[0] * I[1] * I[2]);
                        gA[1] += gm * (double)(I[0] * dA[1] * I[2]);
                        gA[2] += gm * (double)(I[0] * I[1] * dA[2]);
                        gB[0] += gm * (double)(dB[0] * I[1] * I[2]);
                        gB[1] += gm * (double)(I[0] * dB[1] * I[2]);
                        gB[2] += gm * (double)(I[0] * I[1] * dB[2]);
                        gC[0] += gm * (double)(dC[0] * I[1] * I[2]);
                        gC[1] += gm * (double)(I[0] * dC[1] * I[2]);
                        gC[2] += gm * (double)(I[0] * I[1] * dC[2]);
                    }
                }
            }
        }
        const int aA = shell_atom[q.sa], aB = shell_atom[q.sb], aC = shell_atom[q.sc], aD = shell_atom[q.sd];
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            atomicAdd(grad + 3 * aA + x, gA[x]);
            atomicAdd(grad + 3 * aB + x, gB[x]);
            atomicAdd(grad + 3 * aC + x, gC[x]);
            atomicAdd(grad + 3 * aD + x, -(gA[x] + gB[x] + gC[x]));
        }
    }
}

template <typename R>
cudaError_t launch_grad(int qc, const int4 *list, int nq, const PairInfo *pairs, const PrimPair *prims,
                        const double *D, const double *fscale, const int *shell_atom, int n, double *grad,
                        cudaStream_t st, int nsm)
{
    if (nq <= 0) return cudaSuccess;
    int grid = (nq + 127) / 128;
    if (grid > nsm * 32) grid = nsm * 32;
#define PQB_GCASE(CB, CK)                                                                                      \
    case CB *(CB + 1) / 2 + CK:                                                                               \
        eri_grad_kernel<pc_la(CB), pc_lb(CB), pc_la(CK), pc_lb(CK), R>                                         \
            <<<grid, 128, 0, st>>>(list, nq, pairs, prims, D, fscale, shell_atom, n, grad);                   \
        break;
    switch (qc) {
        PQB_GCASE(0, 0)
        PQB_GCASE(1, 0) PQB_GCASE(1, 1)
        PQB_GCASE(2, 0) PQB_GCASE(2, 1) PQB_GCASE(2, 2)
        PQB_GCASE(3, 0) PQB_GCASE(3, 1) PQB_GCASE(3, 2) PQB_GCASE(3, 3)
        PQB_GCASE(4, 0) PQB_GCASE(4, 1) PQB_GCASE(4, 2) PQB_GCASE(4, 3) PQB_GCASE(4, 4)
        PQB_GCASE(5, 0) PQB_GCASE(5, 1) PQB_GCASE(5, 2) PQB_GCASE(5, 3) PQB_GCASE(5, 4) PQB_GCASE(5, 5)
    default:
        return cudaErrorInvalidValue;
    }
#undef PQB_GCASE
    return cudaGetLastError();
}

cudaError_t launch_grad_f64(int qc, const int4 *list, int nq, const PairInfo *pairs, const PrimPair *prims,
                            const double *D, const double *fscale, const int *shell_atom, int n, double *grad,
                            cudaStream_t st, int nsm)
{
    return launch_grad<double>(qc, list, nq, pairs, prims, D, fscale, shell_atom, n, grad, st, nsm);
}

cudaError_t launch_grad_f32(int qc, const int4 *list, int nq, const PairInfo *pairs, const PrimPair *prims,
                            const double *D, const double *fscale, const int *shell_atom, int n, double *grad,
                            cudaStream_t st, int nsm)
{
    return launch_grad<float>(qc, list, nq, pairs, prims, D, fscale, shell_atom, n, grad, st, nsm);
}

}  // namespace pqb
