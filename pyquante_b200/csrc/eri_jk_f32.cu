// Direct J/K instantiations of the ERI engine for the FP32 lists of the mixed
// mode (quartets whose Schwarz bound is below the threshold): integrals and
// per-quartet digestion in single precision, large-T roots and the
// accumulation into J/K in FP64.
#include "eri_engine.cuh"
#include "eri_launch.h"

namespace pqb {
cudaError_t launch_jk_f32(int qc, const int4 *list, int nq, const PairInfo *pairs, const PrimPair *prims,
                          const double *Dscaled, const float *Dscaled_f, double *Jacc, double *Kacc, int n,
                          cudaStream_t st, int nsm, const ItemScreen &scr)
{
    (void)n;
    EpiJK epi{{Dscaled}, {Jacc}, {Kacc}, {Dscaled_f}, scr};
    return launch_eri<float>(qc, list, nq, pairs, prims, epi, st, nsm);
}
}  // namespace pqb
