// Packed-integral instantiations of the ERI engine (FP64).
#include "eri_engine.cuh"
#include "eri_launch.h"

namespace pqb {
cudaError_t launch_packed_f64(int qc, const int4 *list, int nq, const PairInfo *pairs, const PrimPair *prims,
                              double *out, const double *fscale, cudaStream_t st, int nsm)
{
    EpiPacked epi{out, fscale};
    return launch_eri<double>(qc, list, nq, pairs, prims, epi, st, nsm);
}
}  // namespace pqb
