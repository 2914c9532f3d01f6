// Direct J/K instantiations of the ERI engine with FP32 recurrences and
// contraction (roots, weights and prefactors in FP64; digestion into J/K in
// FP64).  Used only for quartets whose Schwarz bound is below the mixed-
// precision threshold.
#include "eri_engine.cuh"
#include "eri_launch.h"

namespace pqb {
cudaError_t launch_jk_f32(int qc, const int4 *list, int nq, const PairInfo *pairs, const PrimPair *prims,
                          const double *Dscaled, double *Jacc, double *Kacc, int n, cudaStream_t st, int nsm)
{
    (void)n;
    EpiJK epi{Dscaled, Jacc, Kacc};
    return launch_eri<float>(qc, list, nq, pairs, prims, epi, st, nsm);
}
}  // namespace pqb
