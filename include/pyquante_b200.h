/* pyquante_b200 — C ABI of the B200 two-electron-integral and Fock-build
 * engine.  Plain C: opaque context, raw device pointers, sizes, int status.
 * No torch or CUDA types appear in the signatures; `stream` is a
 * cudaStream_t passed as void* (NULL = legacy default stream).
 *
 * Every function returns PQB_OK (0) or a PQB_E_* code; the message of the
 * last failure is available from pqb_last_error().  Device buffers are owned
 * by the caller; the context owns only its shell/pair/quartet tables.
 *
 * Reference interfaces replaced (PyQuante, paths inside the project):
 *   - PyQuante/Ints.py:146-167  get2ints      -> pqb_eri_packed
 *   - PyQuante/Ints.py:195-238  getJ/getK/get2JmK on stored integrals
 *                                             -> pqb_jk_packed
 *   - the same three, integral-direct        -> pqb_jk_direct
 *   - PyQuante/Ints.py:73-87    get1ints (S, T+V) -> pqb_oneint
 *   - Src/crys.c:1556-1674 contr_coulomb, :1676-1711 coulomb_repulsion,
 *     Src/cints.c:572-803 (same two), Src/chgp.c:701-890 (contr_coulomb,
 *     hrr, vrr)                                -> pqb_eri_functions
 *   - Src/cints.c:413-425 ijkl2intindex (32-bit; overflows at nbf >= 304)
 *                                             -> pqb_ijkl2intindex (64-bit)
 *   - Src/lib/utils/math.c:27-36 Fgamma (integer m) -> pqb_boys_eval
 *   - Src/crys.c:99-1438 Roots                -> pqb_rys_eval
 */
#ifndef PYQUANTE_B200_H
#define PYQUANTE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    PQB_OK = 0,
    PQB_E_ARG = 1,      /* bad argument (NULL pointer, negative size, ...)   */
    PQB_E_CLASS = 2,    /* angular momentum beyond what the kernels support  */
    PQB_E_NPRIM = 3,    /* too many primitives in one contraction            */
    PQB_E_SHAPE = 4,    /* buffer length does not match the basis            */
    PQB_E_CUDA = 5,     /* a CUDA runtime call failed                        */
    PQB_E_STATE = 6,    /* call order: e.g. no basis uploaded yet            */
    PQB_E_TIMEOUT = 7,  /* a bounded device wait gave up                     */
    PQB_E_NOMEM = 8     /* device (or, in pqb_plan, host) allocation failed  */
};

/* precision modes of pqb_jk_direct */
enum { PQB_FP64 = 0, PQB_MIXED = 1 };
/* engines of pqb_eri_functions */
enum { PQB_ENGINE_RYS = 0, PQB_ENGINE_HGP = 1 };

typedef struct pqb_ctx pqb_ctx;

int pqb_version(void);
int pqb_create(pqb_ctx **ctx, int device);
void pqb_destroy(pqb_ctx *ctx);
/* copies the last error message (NUL-terminated, truncated to len) */
int pqb_last_error(const pqb_ctx *ctx, char *buf, size_t len);

/* Shell basis for the class engine.  Shell s has angular momentum
 * shell_l[s] <= 2 (cartesian, PyQuante component order), shell_nprim[s]
 * primitives starting at prim_off[s] in prim_exp/prim_coef, centre
 * shell_xyz[3s..3s+2] (bohr) and functions [shell_f0[s], shell_f0[s]+ncart).
 * The contracted function f = fscale[f] * sum_p prim_coef[p] * g(alpha_p),
 * g the UNNORMALISED cartesian primitive: prim_coef carries contraction
 * coefficient, primitive norm and contracted norm of the shell's first
 * component; fscale carries each component's ratio to it.  Builds shell
 * pairs and the unscreened quartet lists. */
int pqb_shells_upload(pqb_ctx *ctx, int nshell, const int *shell_l, const int *shell_nprim, const int *prim_off,
                      const int *shell_f0, const double *shell_xyz, const double *prim_exp, const double *prim_coef,
                      int nbf, const double *fscale);

/* Batched basis: nmol molecules, molecule m owning shells
 * [mol_shell_off[m], mol_shell_off[m+1]) and the functions they cover
 * (consecutive).  Shell pairs and quartets never mix molecules; D, J and K
 * of pqb_jk_direct are then the molecules' dense blocks back to back
 * (block m: nm x nm at offset sum_{m'<m} nm'^2, total pqb_dense_len).
 * pqb_shells_upload is the nmol = 1 case.  Packed integrals need nmol = 1. */
int pqb_shells_upload_batch(pqb_ctx *ctx, int nmol, const int *mol_shell_off, int nshell, const int *shell_l,
                            const int *shell_nprim, const int *prim_off, const int *shell_f0, const double *shell_xyz,
                            const double *prim_exp, const double *prim_coef, int nbf, const double *fscale);
int pqb_dense_len(const pqb_ctx *ctx, int64_t *len);
/* Batched basis: a device array of nmol ints; the direct builds
 * (pqb_jk_direct, pqb_jk_direct2) skip the work items of molecules m with
 * mask[m] == 0, whose J and K blocks then come out zero (a batched SCF stops
 * building molecules that have converged).  NULL (the default) builds every
 * molecule.  The array stays owned by the caller and must outlive every
 * build, including builds the caller captured in a CUDA graph; its contents
 * may change between builds.  No counterpart in the reference (one molecule
 * per SCF). */
int pqb_set_molecule_mask(pqb_ctx *ctx, const int *mask);

/* Density screening of the direct builds (incremental Fock builds digest a
 * density difference, most of whose blocks are small): with shell_dmax, a
 * device array of nshell bounds max_ij |D_ij| over each shell's rows i (in
 * its molecule's block; pqb_shell_dmax fills it), a work item (ab|cd) is
 * skipped when Q_ab Q_cd max(dmax[a], dmax[b], dmax[c], dmax[d]) < tau,
 * Q the Schwarz factors of pqb_schwarz (required first).  NULL disables it.
 * The array stays owned by the caller, like the molecule mask; its contents
 * may change between builds.  pqb_shell_dmax writes those bounds for D (the
 * dense layout of pqb_jk_direct) on the stream.  No counterpart in the
 * reference (whose SCF rebuilds F from the full density). */
int pqb_set_density_screen(pqb_ctx *ctx, const double *shell_dmax, double tau);
int pqb_shell_dmax(pqb_ctx *ctx, const double *D, double *shell_dmax, void *stream);

/* One step of canonical purification (Palser and Manolopoulos) for nmat
 * row-major n x n device matrices back to back: from P, P2 = P P and
 * P3 = P2 P, with c = tr(P2 - P3)/tr(P - P2) clamped to [0, 1],
 *   P_out = ((1+c) P2 - P3)/c  (c >= 1/2),  ((1-2c) P + (1+c) P2 - P3)/(1-c)  (else);
 * a matrix with |tr(P - P2)| < tol n is copied unchanged and done[m] = 1
 * (done may be NULL).  P_out may be P; it must not overlap P2 or P3.  The
 * batched and device SCF loops get their densities from this step (GEMMs
 * only, no eigensolver); no counterpart in the reference. */
int pqb_purify_step(int nmat, int n, const double *P, const double *P2, const double *P3, double *P_out, int *done,
                    double tol, void *stream);

/* Schwarz factors Q_ab = sqrt(max |(ab|ab)|) for every shell pair, computed
 * on the device; copied to Q_host (length npairs) when it is not NULL. */
int pqb_schwarz(pqb_ctx *ctx, double *Q_host, void *stream);
int pqb_num_pairs(const pqb_ctx *ctx);

/* Screened quartet plan for pqb_jk_direct: quartets with Q_ab Q_cd <
 * schwarz_thresh are dropped; below fp32_thresh they go to the FP32 list
 * (used in PQB_MIXED mode).  counts (may be NULL) receives
 * {shell quartets, kept FP64, kept FP32, dropped}. */
int pqb_plan(pqb_ctx *ctx, double schwarz_thresh, double fp32_thresh, int64_t *counts);

/* Tuning knobs (used by pyquante_b200.autotune): PQB_PARAM_CHUNK = the
 * largest number of primitive quartets in one J/K work item, for class
 * qclass (0..20, or -1 for all; effective at the next pqb_plan);
 * PQB_PARAM_STREAMS = streams the class launches are spread over (1..16);
 * PQB_PARAM_ORDER = class launch order (0 by estimated cost, 1 highest
 * angular momentum first, the default); PQB_PARAM_PACKED_KERNEL = the
 * stored-integral J/K kernel of pqb_jk_packed (0 automatic: the register
 * form for nbf <= 512, one block per packed row above; 1 always the latter,
 * so tests can compare the two); PQB_PARAM_GRAPH = 1 (default) lets
 * pqb_jk_direct replay a CUDA graph of its class launches, captured on the
 * second call per mode into context-owned accumulators and rebuilt after any
 * change of basis, plan or parameter (single-molecule bases, callers not
 * capturing a graph themselves); 0 launches the classes one by one;
 * PQB_PARAM_THREADS = host threads that pqb_plan enumerates and orders the
 * quartets on (0, the default: all hardware threads up to 32 once a plan
 * has 4M shell quartets or more, else 1); the plan is the same for any
 * count. */
enum { PQB_PARAM_CHUNK = 0, PQB_PARAM_STREAMS = 1, PQB_PARAM_ORDER = 2, PQB_PARAM_PACKED_KERNEL = 3,
       PQB_PARAM_GRAPH = 4, PQB_PARAM_THREADS = 5 };
int pqb_set_param(pqb_ctx *ctx, int param, int qclass, int value);

/* Per-class statistics of the current plan, arrays of 2*21 int64 indexed
 * [part*21 + class] (part 0 = FP64 list, 1 = FP32-eligible list; class =
 * bra*(bra+1)/2 + ket over pair classes ss ps pp ds dp dd): shell quartets and
 * primitive quartets. */
int pqb_plan_stats(const pqb_ctx *ctx, int64_t *quartets, int64_t *prim_quartets);

/* Keep only every nranks-th quartet of each class list of the current plan,
 * starting at rank (multi-GPU sharding of one Fock build). */
int pqb_plan_shard(pqb_ctx *ctx, int rank, int nranks);

/* FP64 FMA throughput probe: `iters` dependent-chain FMA rounds on every SM;
 * returns achieved FP64 FLOP/s in *flops (a roofline denominator). */
int pqb_fp64_peak(pqb_ctx *ctx, int iters, double *flops);

/* All unique (ij|kl), i>=j, k>=l, ij>=kl, at ijkl2intindex (64-bit) into
 * out (device, len = P(P+1)/2, P = nbf(nbf+1)/2).  Unscreened, FP64. */
int pqb_eri_packed(pqb_ctx *ctx, double *out, int64_t len, void *stream);

/* Integral-direct J_ij = sum_kl (ij|kl) D_kl and K_ij = sum_kl (ik|jl) D_kl
 * for a symmetric density D (device, nbf x nbf, row-major); J and K are
 * overwritten.  K may be NULL: then only the Coulomb digestion runs and J
 * alone is written (the getJ of PyQuante/dft.py:209 and :312).
 * mode = PQB_FP64 or PQB_MIXED.  The context's scratch (scaled
 * density, graph accumulators) is shared by its calls: calls on one context
 * must not overlap on different streams (see PQB_PARAM_GRAPH). */
int pqb_jk_direct(pqb_ctx *ctx, const double *D, double *J, double *K, int mode, void *stream);

/* G = 2J - K of a host density in one call: PyQuante's get2JmK(Ints, D)
 * (PyQuante/Ints.py:225-238) on integral-direct integrals, with host arrays
 * D_host and G_host (nbf x nbf, row-major; page-locked for asynchronous
 * copies).  Copies D in, builds as pqb_jk_direct, takes G from the build's
 * accumulators in one pass, and copies G out, all enqueued on the stream:
 * G_host is complete once the stream reaches that point (with a pageable
 * G_host, such as a numpy array, when the call returns: CUDA finishes a
 * device-to-pageable copy before its cudaMemcpyAsync returns).
 * Single-molecule contexts; the context owns the device copies of D and G. */
int pqb_get2jmk_host(pqb_ctx *ctx, const double *D_host, double *G_host, int mode, void *stream);

/* J and K of two densities from one pass over the integrals: every
 * integral is evaluated once and digested against Da and Db.  Replaces the
 * four calls getJ(Ints, Da), getJ(Ints, Db), getK(Ints, Da), getK(Ints, Db)
 * of the reference's UHF iteration (PyQuante/hartree_fock.py:233-236, the
 * same pattern in PyQuante2.py:200-202 and rohf.py:332-335).  Same rules as
 * pqb_jk_direct for each density. */
int pqb_jk_direct2(pqb_ctx *ctx, const double *Da, const double *Db, double *Ja, double *Ka, double *Jb, double *Kb,
                   int mode, void *stream);

/* One class list of the plan only (part 0 FP64 list / 1 FP32-eligible list,
 * class 0..20), accumulating unsymmetrised contributions into Jacc/Kacc
 * (not cleared).  The contributions are those of the element-scaled density
 * D_kl r_k r_l (r = the per-function scales of pqb_shells_upload); the full
 * pqb_jk_direct applies r_i r_j to J and K.  For per-class timing and tuning. */
int pqb_jk_direct_class(pqb_ctx *ctx, const double *D, double *Jacc, double *Kacc, int part, int qclass, int mode,
                        void *stream);

/* AO -> MO transformation for MP2 (replaces the Python loops of
 * PyQuante/MP.py:20-75 TransformIntsMP2 and :77-97 MP2).  The quarter
 * transformations are FP64 GEMMs the caller runs (cuBLAS); these move the
 * data between them.  All pointers are device memory; no context.
 * pqb_mo_unpack_rows: out[r][k][l] = (IJ|kl) for the packed bra rows
 *   IJ = row0 .. row0+nrows-1 of the packed array ints (len = P(P+1)/2,
 *   P = nbf(nbf+1)/2): out holds nrows * nbf * nbf doubles.
 * pqb_mo_unpack_pairs: out[(mu*nbf + nu)*ncol + c] = Y[pair(mu,nu)*ncol + c]
 *   (rows stored per packed AO pair, unpacked to both orders).
 * pqb_mo_pack: moints[ijkl2intindex(a,i,b,j)] = Z[((a*nmo + i)*nocc + b)*nmo + j]
 *   for a, b < nocc, i, j < nmo (len = Q(Q+1)/2, Q = nmo(nmo+1)/2: the
 *   packed MO array TransformIntsMP2 returns; other slots are left as is).
 * pqb_mp2_pairs: Epair[a*nocc + b] = sum_rs (ar|bs)(2(ar|bs) - (as|br)) /
 *   (e_a + e_b - e_r - e_s) from V[((a*nvirt + r)*nocc + b)*nvirt + s]. */
int pqb_mo_unpack_rows(const double *ints, int64_t len, int nbf, int64_t row0, int nrows, double *out, void *stream);
int pqb_mo_unpack_pairs(const double *Y, int nbf, int64_t ncol, double *out, void *stream);
int pqb_mo_pack(const double *Z, int nocc, int nmo, double *moints, int64_t len, void *stream);
int pqb_mp2_pairs(const double *V, int nocc, int nvirt, const double *e_occ, const double *e_virt, double *Epair,
                  void *stream);

/* DFT numerical integration (replaces the Python loops of the reference's
 * MG2 grid and SVWN functional: PyQuante/MG2.py:50-250,
 * PyQuante/MolecularGrid.py:228-263, PyQuante/DFunctionals.py:76-138,
 * 319-389, 603-623, and the Fxc assembly of PyQuante/dft.py:29-65).  All
 * pointers are device memory; no context.
 * pqb_becke_weights: w[g] = pts[4g+3] * P_owner / sum_j P_j for the points
 *   pts[npts][4] (x, y, z, atomic-grid weight), owner[g] its atom,
 *   atom_xyz[3*natoms], adjust[natoms*natoms] the heteronuclear size
 *   adjustment a_jk (mu' = mu + a_jk (1 - mu^2)).
 * pqb_grid_amps: B[g*n + i] = amplitude of basis function i (the function
 *   table of pqb_oneint) at point g of pts[npts][4].
 * pqb_grid_rowdot: out[g] = sum_i A[g*n + i] B[g*n + i] (the density from
 *   B D and B).
 * pqb_xc_svwn: per point, Slater exchange plus VWN correlation of the spin
 *   densities rhoa, rhob, times the weight w: wf = w f_xc, wva = w v_a,
 *   wvb = w v_b. */
int pqb_becke_weights(int npts, const double *pts, const int *owner, int natoms, const double *atom_xyz,
                      const double *adjust, double *w, void *stream);
int pqb_grid_amps(int n, const double *origin, const int *powers, const int *prim_off, const double *exps,
                  const double *cn, const double *norms, int npts, const double *pts, double *B, void *stream);
int pqb_grid_rowdot(int npts, int n, const double *A, const double *B, double *out, void *stream);
int pqb_xc_svwn(int npts, const double *rhoa, const double *rhob, const double *w, double *wf, double *wva,
                double *wvb, void *stream);

/* The same J and K from stored packed integrals (device). */
int pqb_jk_packed(pqb_ctx *ctx, const double *ints, int64_t len, const double *D, double *J, double *K, int nbf,
                  void *stream);

/* Stateless per-function kernels over a device function table:
 * origin[3n], powers[3n], prim_off[n+1], exps/cn[prim_off[n]] where
 * cn = contraction coefficient * primitive norm, norms[n] (contracted norm).
 * pqb_eri_functions: out[q] = norms_a..d * sum cn_a..cn_d (prim ERI) for the
 * function quartets quartets[4q..4q+3] (total angular momentum <= 9), by Rys
 * quadrature (PQB_ENGINE_RYS) or Head-Gordon--Pople (PQB_ENGINE_HGP;
 * |a|+|b| <= 4 and |c|+|d| <= 4).  aux_m > 0 (HGP only) returns the
 * auxiliary (ab|cd)^(m) of chgp.vrr (Src/chgp.c:244-419) instead.
 * pqb_oneint: S, T, V (each n x n, any may be NULL) with V = sum_atoms Z_a
 * <i|-1/|r-R_a||j>. */
int pqb_eri_functions(pqb_ctx *ctx, int engine, int aux_m, int nq, const int *quartets, int n, const double *origin,
                      const int *powers, const int *prim_off, const double *exps, const double *cn,
                      const double *norms, double *out, void *stream);
int pqb_oneint(pqb_ctx *ctx, int n, const double *origin, const int *powers, const int *prim_off, const double *exps,
               const double *cn, const double *norms, int natoms, const double *atom_xyz, const double *atom_z,
               double *S, double *T, double *V, void *stream);

/* Allocation-free variant of pqb_oneint, for callers that may not allocate
 * device memory: code running where a framework's memory pool owns the GPU,
 * inside a region that must not trigger allocation, or with a fixed memory
 * budget.  No counterpart in the reference.  Differences from pqb_oneint:
 * no context argument, atom_xyz[3*natoms] and atom_z[natoms] are DEVICE
 * arrays, and the packed atom table the kernel reads lives in a file-scope
 * device array of PQB_NOALLOC_MAX_ATOMS = 4096 atoms (128 KiB per GPU, held
 * until exit); natoms above that returns PQB_E_SHAPE.  It calls no
 * cudaMalloc/cudaFree.  The atoms are read only when V is requested (V may
 * be NULL, as in pqb_oneint).  `stream` must belong to the current device
 * (PQB_E_ARG otherwise).  The first call on each device that computes V
 * looks the array's address up (cudaGetSymbolAddress, that device current);
 * make that first call before any stream capture.  All calls share the
 * array: calls that overlap on the GPU (e.g. on two streams) race; each call
 * rewrites the entries it uses, so nothing needs clearing.  Status codes
 * only (no context, so no pqb_last_error message). */
int pqb_oneint_noalloc(int n, const double *origin, const int *powers, const int *prim_off, const double *exps,
                       const double *cn, const double *norms, int natoms, const double *atom_xyz,
                       const double *atom_z, double *S, double *T, double *V, void *stream);

/* RHF nuclear gradient (replaces PyQuante/force.py:48-70 with
 * AnalyticDerivatives.py): dE/dR = 2 tr(D dh) + tr(D dG[D]) - 2 tr(W dS)
 * + dE_nuc, D = C_occ C_occ^T, W = C_occ diag(e_occ) C_occ^T.
 * pqb_set_shell_atoms: atom index of every uploaded shell (host array).
 * pqb_grad_2e: adds tr(D dG[D]) to grad[3*natoms] (device), derivative
 * integrals contracted with the density on the fly over the current plan;
 * mode PQB_MIXED runs the FP32-eligible list in FP32.
 * pqb_grad_1e: adds 2 tr(D d(T+V)) - 2 tr(W dS) over a function table
 * (func_atom: device array, atom index per function; atoms on the host). */
int pqb_set_shell_atoms(pqb_ctx *ctx, const int *shell_atom);
int pqb_grad_2e(pqb_ctx *ctx, const double *D, double *grad, int mode, void *stream);
int pqb_grad_1e(pqb_ctx *ctx, int n, const double *origin, const int *powers, const int *prim_off, const double *exps,
                const double *cn, const double *norms, const int *func_atom, int natoms, const double *atom_xyz,
                const double *atom_z, const double *D, const double *W, double *grad, void *stream);

/* Canonical packed index, 64-bit. */
int64_t pqb_ijkl2intindex(int64_t i, int64_t j, int64_t k, int64_t l);

/* Kernel-level checks: F_0..F_m(T_i) into F[i*(m+1)+k] (m <= 16), and the
 * n-root Rys rule (n <= 5) at T_i into u[i*n+r], w[i*n+r].  Device arrays.
 * pqb_boys_rows_eval: F_0..F_lt (lt <= 4) by the form the thread-mode
 * Fock-build kernels use (compact Taylor rows, large-T asymptotics, no
 * branches), into F[i*(lt+1)+k]. */
int pqb_boys_eval(pqb_ctx *ctx, int m, int count, const double *T, double *F, void *stream);
int pqb_boys_rows_eval(pqb_ctx *ctx, int lt, int count, const double *T, double *F, void *stream);
int pqb_rys_eval(pqb_ctx *ctx, int nroots, int count, const double *T, double *u, double *w, void *stream);

#ifdef __cplusplus
}
#endif
#endif
