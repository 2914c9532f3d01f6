// Schwarz-bound instantiations of the ERI engine (diagonal quartets, FP64).
#include "eri_engine.cuh"
#include "eri_launch.h"

namespace pqb {
cudaError_t launch_schwarz_f64(int qc, const int4 *list, int nq, const PairInfo *pairs, const PrimPair *prims,
                               unsigned long long *Q2bits, const double *fscale, cudaStream_t st, int nsm)
{
    EpiSchwarz epi{Q2bits, fscale};
    return launch_eri<double>(qc, list, nq, pairs, prims, epi, st, nsm);
}
}  // namespace pqb
