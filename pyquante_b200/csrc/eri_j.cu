// Coulomb-only direct builds (J without K: the getJ of the DFT path) of the
// ERI engine, FP64 integrals and the FP32 lists of the mixed mode.
#include "eri_engine.cuh"
#include "eri_launch.h"

namespace pqb {
cudaError_t launch_j_f64(int qc, const int4 *list, int nq, const PairInfo *pairs, const PrimPair *prims,
                         const double *Dscaled, double *Jacc, cudaStream_t st, int nsm, const ItemScreen &scr)
{
    EpiJ epi{{Dscaled}, {Jacc}, {nullptr}, {nullptr}, scr};
    return launch_eri<double>(qc, list, nq, pairs, prims, epi, st, nsm);
}

cudaError_t launch_j_f32(int qc, const int4 *list, int nq, const PairInfo *pairs, const PrimPair *prims,
                         const double *Dscaled, const float *Dscaled_f, double *Jacc, cudaStream_t st, int nsm,
                         const ItemScreen &scr)
{
    EpiJ epi{{Dscaled}, {Jacc}, {nullptr}, {Dscaled_f}, scr};
    return launch_eri<float>(qc, list, nq, pairs, prims, epi, st, nsm);
}
}  // namespace pqb
