// Device-resident data layout of a basis (built by the host in pqb_capi.cu).
//
// Shell pairs are stored once per unordered pair of shells, oriented so the
// first shell has the higher angular momentum (ties: higher shell index);
// the Rys horizontal transfer moves momentum from the first to the second.
// Each pair owns a run of primitive pairs with the Gaussian-product data.
#pragma once
#include <stdint.h>

namespace pqb {

constexpr int kMaxL = 2;                         // shells up to d (cartesian)
constexpr int kNumPairClass = 6;                 // ss ps pp ds dp dd
constexpr int kNumQuartetClass = 21;             // bra class >= ket class

// Per-item screening of the direct builds (all fields optional):
//   molmask: batched bases, molecule m's items are skipped when molmask[m] == 0;
//   dmax:    per shell, a bound on |D_ij| over the shell's rows i (within
//            its molecule's block); an item (ab|cd) is skipped when
//            Q_ab Q_cd max(dmax[a], dmax[b], dmax[c], dmax[d]) < tau, Q the
//            Schwarz factors (the incremental builds of a batched SCF digest
//            density differences, most of which are small).
struct ItemScreen {
    const int *molmask;
    const double *dmax;
    const double *Qpair;
    double tau;
};

struct PairInfo {
    double A[3];       // centre of the first shell
    double AB[3];      // A - B
    int prim_off;      // first PrimPair
    int nprim;         // number of (screened) primitive pairs
    int fa, fb;        // first basis-function index of each shell
    int sa, sb;        // shell indices
    int cls;           // pair class: index of (La, Lb) in ss ps pp ds dp dd
    int la, lb;
    int nm;            // functions of the pair's molecule (batched bases; else nbf)
    int mol;           // the pair's molecule (batched bases; else 0)
    long long bo;      // D/J/K element (i, j) of the molecule is at bo + i*nm + j
                       // (global function indices; 0 for a single molecule)
};

// 96 bytes, 32-byte aligned.  The FP64 kernels fetch the Fock-build fields
// with one 256-bit and one 128-bit load; the FP32 kernels (mixed precision)
// fetch their single-precision copy, f[], with one 256-bit load.
struct __align__(32) PrimPair {
    double zeta;       // alpha_a + alpha_b
    double izeta;      // 1 / zeta (the recurrences multiply; no division per quartet)
    double P[3];       // Gaussian product centre
    double K;          // c_a c_b sqrt(2) pi^(5/4)/zeta exp(-alpha_a alpha_b/zeta |AB|^2)
    double alpha_a;    // exponent of the first shell's primitive (alpha_b = zeta - alpha_a)
    double pad_;
    float f[8];        // zeta, 1/zeta, P[3], K rounded to single precision, 0, 0
};

__host__ __device__ inline int pair_class(int la, int lb)   // la >= lb
{
    return la * (la + 1) / 2 + lb;
}

// quartet class index for bra class cb >= ket class ck
__host__ __device__ inline int quartet_class(int cb, int ck) { return cb * (cb + 1) / 2 + ck; }

}  // namespace pqb
