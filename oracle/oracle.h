/* CPU oracle (test infrastructure only; never linked into the product).
 *
 * A plain-C restatement of the reference's integral path:
 *   - two-electron integrals by the Head-Gordon--Pople scheme of
 *     Src/chgp.c:78-419 (contracted HRR b->a, d->c over an Obara--Saika VRR),
 *     with the Boys function evaluated to long-double accuracy instead of the
 *     reference's Numerical-Recipes incomplete gamma (EPS 3e-7,
 *     Src/chgp.c:35-37,619-690), so the oracle agrees with the reference's
 *     FP64-faithful Rys engine (Src/crys.c) to ~1e-14;
 *   - one-electron integrals by the THO formulas of Src/cints.c:190-307;
 *   - the get2ints loop and packing of PyQuante/Ints.py:146-167 with the
 *     index of Src/cints.c:413-425 in 64 bits;
 *   - getJ/getK/get2JmK of PyQuante/Ints.py:195-238.
 */
#ifndef PQB_ORACLE_H
#define PQB_ORACLE_H
#include <stdint.h>

double orc_boys(int m, double T);
int64_t orc_ijkl2intindex(int64_t i, int64_t j, int64_t k, int64_t l);

double orc_prim_eri(const double *A, double na, const int *la, double aa,
                    const double *B, double nb, const int *lb, double ab,
                    const double *C, double nc, const int *lc, double ac,
                    const double *D, double nd, const int *ld, double ad);

double orc_contr_eri(int lena, const double *aexps, const double *acoefs, const double *anorms,
                     const double *A, const int *la,
                     int lenb, const double *bexps, const double *bcoefs, const double *bnorms,
                     const double *B, const int *lb,
                     int lenc, const double *cexps, const double *ccoefs, const double *cnorms,
                     const double *C, const int *lc,
                     int lend, const double *dexps, const double *dcoefs, const double *dnorms,
                     const double *D, const int *ld);

int orc_get2ints(int64_t nbf, const double *origin, const int64_t *powers, const int64_t *prim_off,
                 const double *exps, const double *coefs, const double *pnorms, const double *norms,
                 double *out);

void orc_get1ints(int64_t nbf, const double *origin, const int64_t *powers, const int64_t *prim_off,
                  const double *exps, const double *coefs, const double *pnorms, const double *norms,
                  int64_t natoms, const double *atom_xyz, const double *atom_z, double *S, double *h);

void orc_getJK(int64_t nbf, const double *ints, const double *D, double *J, double *K);
#endif
