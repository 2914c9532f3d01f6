// AO -> MO integral transformation for the MP2 energy (the work of the
// reference's PyQuante/MP.py:20-75 TransformIntsMP2 and :77-97 MP2), on
// the packed integrals of pqb_eri_packed.
//
// The four quarter transformations are dense FP64 contractions and run as
// cuBLAS DGEMMs from the host side; the kernels here move the data between
// them without storing anything twice:
//   * mo_unpack_rows_kernel: a batch of packed bra rows (ij| into dense
//     N x N matrices (ij|kl), for every kl (the gather of the 8-fold packed
//     order, Src/cints.c:413-425, in 64 bits);
//   * mo_unpack_pairs_kernel: half-transformed integrals stored per packed
//     AO pair back into dense (mu, nu) rows, symmetric;
//   * mo_pack_kernel: (ai|bj) into the reference's packed MO array at
//     ijkl2intindex(a, i, b, j);
//   * mp2_pairs_kernel: the pair energies
//       E_ab = sum_rs (ar|bs) (2 (ar|bs) - (as|br)) / (e_a + e_b - e_r - e_s).
#include <cstdint>

#include <cuda_runtime.h>

#include "../../include/pyquante_b200.h"

namespace {

__device__ __forceinline__ int64_t pair_of(int64_t i, int64_t j)
{
    return i >= j ? i * (i + 1) / 2 + j : j * (j + 1) / 2 + i;
}

__device__ __forceinline__ int64_t packed_of(int64_t ij, int64_t kl)
{
    return ij >= kl ? ij * (ij + 1) / 2 + kl : kl * (kl + 1) / 2 + ij;
}

// out[r][k][l] = (IJ_r|kl), IJ_r = row0 + r.  One thread per output element
// (writes coalesced; the reads are the packed rows, contiguous for kl <= IJ
// and strided by kl beyond).
__global__ void mo_unpack_rows_kernel(const double *__restrict__ ints, int nbf, int64_t row0, int nrows,
                                      double *__restrict__ out)
{
    const int64_t nn = (int64_t)nbf * nbf, total = nn * nrows;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = t / nn, kl = t - r * nn;
        const int64_t k = kl / nbf, l = kl - k * nbf;
        out[t] = __ldg(ints + packed_of(row0 + r, pair_of(k, l)));
    }
}

// out[(mu * nbf + nu) * ncol + c] = Y[pair(mu, nu) * ncol + c].
__global__ void mo_unpack_pairs_kernel(const double *__restrict__ Y, int nbf, int64_t ncol, double *__restrict__ out)
{
    const int64_t total = (int64_t)nbf * nbf * ncol;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t row = t / ncol, c = t - row * ncol;
        const int64_t mu = row / nbf, nu = row - mu * nbf;
        out[t] = __ldg(Y + pair_of(mu, nu) * ncol + c);
    }
}

// moints[ijkl2intindex(a, i, b, j)] = Z[((a * nmo + i) * nocc + b) * nmo + j]
// for a, b < nocc, i, j < nmo.  Slots that several (a, i, b, j) share by
// symmetry receive the same integral.
__global__ void mo_pack_kernel(const double *__restrict__ Z, int nocc, int nmo, double *__restrict__ moints)
{
    const int64_t total = (int64_t)nocc * nmo * nocc * nmo;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        int64_t q = t;
        const int64_t j = q % nmo;
        q /= nmo;
        const int64_t b = q % nocc;
        q /= nocc;
        const int64_t i = q % nmo, a = q / nmo;
        moints[packed_of(pair_of(a, i), pair_of(b, j))] = Z[t];
    }
}

// One block per occupied pair (a, b): V[((a * nv + r) * nocc + b) * nv + s]
// = (ar|bs) over the virtual orbitals r, s.
__global__ void __launch_bounds__(256) mp2_pairs_kernel(const double *__restrict__ V, int nocc, int nv,
                                                        const double *__restrict__ e_occ,
                                                        const double *__restrict__ e_virt, double *__restrict__ Epair)
{
    const int a = blockIdx.x / nocc, b = blockIdx.x - a * nocc;
    const double eab = e_occ[a] + e_occ[b];
    double sum = 0.0;
    for (int t = threadIdx.x; t < nv * nv; t += blockDim.x) {
        const int r = t / nv, s = t - r * nv;
        const double v = V[(((int64_t)a * nv + r) * nocc + b) * nv + s];
        const double w = V[(((int64_t)a * nv + s) * nocc + b) * nv + r];
        sum += v * (2.0 * v - w) / (eab - e_virt[r] - e_virt[s]);
    }
    __shared__ double red[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sum;
    __syncthreads();
    if (threadIdx.x < 32) {
        sum = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_down_sync(0xffffffffu, sum, o);
        if (threadIdx.x == 0) Epair[blockIdx.x] = sum;
    }
}

int grid_for(int64_t total)
{
    const int64_t g = (total + 255) / 256;
    return (int)(g < 148 * 32 ? (g > 0 ? g : 1) : 148 * 32);
}

}  // namespace

extern "C" {

int pqb_mo_unpack_rows(const double *ints, int64_t len, int nbf, int64_t row0, int nrows, double *out, void *stream)
{
    if (!ints || !out || nbf <= 0 || nrows <= 0 || row0 < 0) return PQB_E_ARG;
    const int64_t P = (int64_t)nbf * (nbf + 1) / 2;
    if (len != P * (P + 1) / 2 || row0 + nrows > P) return PQB_E_SHAPE;
    const int64_t total = (int64_t)nbf * nbf * nrows;
    mo_unpack_rows_kernel<<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(ints, nbf, row0, nrows, out);
    return cudaGetLastError() == cudaSuccess ? PQB_OK : PQB_E_CUDA;
}

int pqb_mo_unpack_pairs(const double *Y, int nbf, int64_t ncol, double *out, void *stream)
{
    if (!Y || !out || nbf <= 0 || ncol <= 0) return PQB_E_ARG;
    const int64_t total = (int64_t)nbf * nbf * ncol;
    mo_unpack_pairs_kernel<<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(Y, nbf, ncol, out);
    return cudaGetLastError() == cudaSuccess ? PQB_OK : PQB_E_CUDA;
}

int pqb_mo_pack(const double *Z, int nocc, int nmo, double *moints, int64_t len, void *stream)
{
    if (!Z || !moints || nocc <= 0 || nmo <= 0 || nocc > nmo) return PQB_E_ARG;
    const int64_t P = (int64_t)nmo * (nmo + 1) / 2;
    if (len != P * (P + 1) / 2) return PQB_E_SHAPE;
    const int64_t total = (int64_t)nocc * nmo * nocc * nmo;
    mo_pack_kernel<<<grid_for(total), 256, 0, (cudaStream_t)stream>>>(Z, nocc, nmo, moints);
    return cudaGetLastError() == cudaSuccess ? PQB_OK : PQB_E_CUDA;
}

int pqb_mp2_pairs(const double *V, int nocc, int nvirt, const double *e_occ, const double *e_virt, double *Epair,
                  void *stream)
{
    if (!V || !e_occ || !e_virt || !Epair || nocc <= 0 || nvirt < 0) return PQB_E_ARG;
    if (nvirt == 0) return cudaMemsetAsync(Epair, 0, sizeof(double) * nocc * nocc, (cudaStream_t)stream) ==
                                   cudaSuccess ? PQB_OK : PQB_E_CUDA;
    mp2_pairs_kernel<<<nocc * nocc, 256, 0, (cudaStream_t)stream>>>(V, nocc, nvirt, e_occ, e_virt, Epair);
    return cudaGetLastError() == cudaSuccess ? PQB_OK : PQB_E_CUDA;
}

}  // extern "C"
