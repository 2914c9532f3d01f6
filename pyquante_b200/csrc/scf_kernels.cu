// Dense SCF step kernels of the batched and device SCF loops (no
// counterpart in the reference, whose SCF diagonalises on the host):
//   * purify_step_kernel: one step of the canonical purification of Palser
//     and Manolopoulos (Phys. Rev. B 58, 12704 (1998)) for a batch of
//     matrices, given P, P^2 and P^3 (two library GEMMs before it):
//       c = tr(P^2 - P^3) / tr(P - P^2), clamped to [0, 1];
//       P' = ((1+c) P^2 - P^3) / c             for c >= 1/2,
//       P' = ((1-2c) P + (1+c) P^2 - P^3) / (1-c)  otherwise;
//     a matrix already idempotent to rounding (|tr(P - P^2)| < tol n) is
//     kept and flagged done.  One block per matrix: the traces by a block
//     reduction, then the update, in one launch (the elementwise form in
//     tensor operations takes some fifteen launches per step).
#include <cstdint>

#include <cuda_runtime.h>

#include "../../include/pyquante_b200.h"

namespace {

constexpr int kPurifyThreads = 256;

__global__ void __launch_bounds__(kPurifyThreads) purify_step_kernel(int n, const double *__restrict__ P,
                                                                   const double *__restrict__ P2,
                                                                   const double *__restrict__ P3,
                                                                   double *__restrict__ Pout, int *__restrict__ done,
                                                                   double tol)
{
    const int64_t off = (int64_t)blockIdx.x * n * n;
    const double *p = P + off, *p2 = P2 + off, *p3 = P3 + off;
    double *po = Pout + off;
    __shared__ double s_num[kPurifyThreads / 32], s_den[kPurifyThreads / 32];
    double num = 0.0, den = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int64_t ii = (int64_t)i * n + i;
        num += p2[ii] - p3[ii];
        den += p[ii] - p2[ii];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        num += __shfl_xor_sync(0xffffffffu, num, o);
        den += __shfl_xor_sync(0xffffffffu, den, o);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        s_num[warp] = num;
        s_den[warp] = den;
    }
    __syncthreads();
    num = 0.0;
    den = 0.0;
#pragma unroll
    for (int w = 0; w < kPurifyThreads / 32; ++w) {
        num += s_num[w];
        den += s_den[w];
    }
    const bool fin = fabs(den) < tol * n;
    double c = fin ? 0.5 : num / den;
    c = c < 0.0 ? 0.0 : (c > 1.0 ? 1.0 : c);
    const bool hi = c >= 0.5;
    const double a0 = hi ? 0.0 : (1.0 - 2.0 * c), a1 = 1.0 + c;
    const double inv = 1.0 / (hi ? (c > 1e-300 ? c : 1e-300) : ((1.0 - c) > 1e-300 ? (1.0 - c) : 1e-300));
    const int64_t nn = (int64_t)n * n;
    for (int64_t e = threadIdx.x; e < nn; e += blockDim.x) {
        const double x = p[e];
        po[e] = fin ? x : fma(a0, x, fma(a1, p2[e], -p3[e])) * inv;
    }
    if (threadIdx.x == 0 && done) done[blockIdx.x] = fin ? 1 : 0;
}

}  // namespace

extern "C" {

int pqb_purify_step(int nmat, int n, const double *P, const double *P2, const double *P3, double *P_out, int *done,
                    double tol, void *stream)
{
    if (nmat < 0 || n <= 0 || !P || !P2 || !P3 || !P_out) return PQB_E_ARG;
    if (nmat == 0) return PQB_OK;
    purify_step_kernel<<<nmat, kPurifyThreads, 0, (cudaStream_t)stream>>>(n, P, P2, P3, P_out, done, tol);
    return cudaGetLastError() == cudaSuccess ? PQB_OK : PQB_E_CUDA;
}

}  // extern "C"
