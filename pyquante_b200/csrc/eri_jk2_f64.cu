// Two-density direct J/K instantiations of the ERI engine (FP64 integrals):
// UHF's alpha and beta densities digest every integral of one pass.
#include "eri_engine.cuh"
#include "eri_launch.h"

namespace pqb {
cudaError_t launch_jk2_f64(int qc, const int4 *list, int nq, const PairInfo *pairs, const PrimPair *prims,
                           const double *const Dscaled[2], double *const Jacc[2], double *const Kacc[2],
                           cudaStream_t st, int nsm, const ItemScreen &scr)
{
    EpiJK2 epi{{Dscaled[0], Dscaled[1]}, {Jacc[0], Jacc[1]}, {Kacc[0], Kacc[1]}, {nullptr, nullptr}, scr};
    return launch_eri<double>(qc, list, nq, pairs, prims, epi, st, nsm);
}
}  // namespace pqb
