// Direct J/K instantiations of the ERI engine (FP64 integrals).
#include "eri_engine.cuh"
#include "eri_launch.h"

namespace pqb {
cudaError_t launch_jk_f64(int qc, const int4 *list, int nq, const PairInfo *pairs, const PrimPair *prims,
                          const double *Dscaled, double *Jacc, double *Kacc, int n, cudaStream_t st, int nsm,
                          const ItemScreen &scr)
{
    (void)n;
    EpiJK epi{{Dscaled}, {Jacc}, {Kacc}, {nullptr}, scr};
    return launch_eri<double>(qc, list, nq, pairs, prims, epi, st, nsm);
}
}  // namespace pqb
