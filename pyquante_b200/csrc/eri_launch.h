// Work items are int4 {bra pair, ket pair, first primitive quartet, count}:
// a shell quartet's primitive quartets (bra-major, ket-minor) may be split
// over several items whose contributions add (J/K digestion is linear).
// Host-side entry points into the class-templated ERI engine (the direct J/K
// ones take the pre-scaled density D'_kl = r_k r_l D_kl, see EpiJK, and an
// optional item screen, see ItemScreen), one per
// (epilogue, precision) combination; each lives in its own translation unit
// so the 21 class instantiations compile in parallel.
#pragma once
#include <cuda_runtime.h>

#include "pqb_types.h"

namespace pqb {
struct EpiPacked;
template <int NDEN, bool WITHK> struct EpiJKn;
struct EpiSchwarz;

cudaError_t launch_packed_f64(int qc, const int4 *list, int nq, const PairInfo *pairs, const PrimPair *prims,
                              double *out, const double *fscale, cudaStream_t st, int nsm);
cudaError_t launch_jk_f64(int qc, const int4 *list, int nq, const PairInfo *pairs, const PrimPair *prims,
                          const double *Dscaled, double *Jacc, double *Kacc, int n, cudaStream_t st, int nsm,
                          const ItemScreen &scr = ItemScreen{});
cudaError_t launch_jk_f32(int qc, const int4 *list, int nq, const PairInfo *pairs, const PrimPair *prims,
                          const double *Dscaled, const float *Dscaled_f, double *Jacc, double *Kacc, int n,
                          cudaStream_t st, int nsm, const ItemScreen &scr = ItemScreen{});
// J alone (the Coulomb digestion, no exchange)
cudaError_t launch_j_f64(int qc, const int4 *list, int nq, const PairInfo *pairs, const PrimPair *prims,
                         const double *Dscaled, double *Jacc, cudaStream_t st, int nsm, const ItemScreen &scr = ItemScreen{});
cudaError_t launch_j_f32(int qc, const int4 *list, int nq, const PairInfo *pairs, const PrimPair *prims,
                         const double *Dscaled, const float *Dscaled_f, double *Jacc, cudaStream_t st, int nsm,
                         const ItemScreen &scr = ItemScreen{});
// two densities (UHF alpha and beta) digesting the same integrals
cudaError_t launch_jk2_f64(int qc, const int4 *list, int nq, const PairInfo *pairs, const PrimPair *prims,
                           const double *const Dscaled[2], double *const Jacc[2], double *const Kacc[2],
                           cudaStream_t st, int nsm, const ItemScreen &scr = ItemScreen{});
cudaError_t launch_jk2_f32(int qc, const int4 *list, int nq, const PairInfo *pairs, const PrimPair *prims,
                           const double *const Dscaled[2], const float *const Dscaled_f[2], double *const Jacc[2],
                           double *const Kacc[2], cudaStream_t st, int nsm, const ItemScreen &scr = ItemScreen{});
cudaError_t launch_schwarz_f64(int qc, const int4 *list, int nq, const PairInfo *pairs, const PrimPair *prims,
                               unsigned long long *Q2bits, const double *fscale, cudaStream_t st, int nsm);
cudaError_t launch_grad_f64(int qc, const int4 *list, int nq, const PairInfo *pairs, const PrimPair *prims,
                            const double *D, const double *fscale, const int *shell_atom, int n, double *grad,
                            cudaStream_t st, int nsm);
cudaError_t launch_grad_f32(int qc, const int4 *list, int nq, const PairInfo *pairs, const PrimPair *prims,
                            const double *D, const double *fscale, const int *shell_atom, int n, double *grad,
                            cudaStream_t st, int nsm);
}  // namespace pqb
