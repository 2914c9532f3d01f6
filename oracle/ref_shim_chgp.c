/* Test-infrastructure shim: compiles the reference's Src/chgp.c (HGP engine)
 * unmodified, from the reference tree, and exports plain-C entry points for
 * ctypes.  The CPython module-init call (Src/chgp.c:903) is neutralised; no
 * Python object is ever created.  Output goes to oracle/_ref/ only.          */
#define Py_InitModule(n, m) ((void *)0)
#include "Src/chgp.c"

/* chgp.coulomb_repulsion == hrr (Src/chgp.c:172-242, bound at :895) */
double ref_chgp_hrr(double xa, double ya, double za, double norma, int la, int ma, int na, double alphaa,
                    double xb, double yb, double zb, double normb, int lb, int mb, int nb, double alphab,
                    double xc, double yc, double zc, double normc, int lc, int mc, int nc, double alphac,
                    double xd, double yd, double zd, double normd, int ld, int md, int nd, double alphad)
{
    return hrr(xa, ya, za, norma, la, ma, na, alphaa, xb, yb, zb, normb, lb, mb, nb, alphab,
               xc, yc, zc, normc, lc, mc, nc, alphac, xd, yd, zd, normd, ld, md, nd, alphad);
}

/* chgp.vrr (Src/chgp.c:244-419, bound at :896) */
double ref_chgp_vrr(double xa, double ya, double za, double norma, int la, int ma, int na, double alphaa,
                    double xb, double yb, double zb, double normb, double alphab,
                    double xc, double yc, double zc, double normc, int lc, int mc, int nc, double alphac,
                    double xd, double yd, double zd, double normd, double alphad, int m)
{
    return vrr(xa, ya, za, norma, la, ma, na, alphaa, xb, yb, zb, normb, alphab,
               xc, yc, zc, normc, lc, mc, nc, alphac, xd, yd, zd, normd, alphad, m);
}

/* chgp.contr_coulomb (Src/chgp.c:701-818 -> contr_hrr :78-145).  Argument
 * order follows the Python binding: exps, coefs, norms, origin, powers.      */
double ref_chgp_contr(int lena, const double *aexps, const double *acoefs, const double *anorms,
                      const double *xyza, const int *lmna,
                      int lenb, const double *bexps, const double *bcoefs, const double *bnorms,
                      const double *xyzb, const int *lmnb,
                      int lenc, const double *cexps, const double *ccoefs, const double *cnorms,
                      const double *xyzc, const int *lmnc,
                      int lend, const double *dexps, const double *dcoefs, const double *dnorms,
                      const double *xyzd, const int *lmnd)
{
    return contr_hrr(lena, xyza[0], xyza[1], xyza[2], (double *)anorms, lmna[0], lmna[1], lmna[2],
                     (double *)aexps, (double *)acoefs,
                     lenb, xyzb[0], xyzb[1], xyzb[2], (double *)bnorms, lmnb[0], lmnb[1], lmnb[2],
                     (double *)bexps, (double *)bcoefs,
                     lenc, xyzc[0], xyzc[1], xyzc[2], (double *)cnorms, lmnc[0], lmnc[1], lmnc[2],
                     (double *)cexps, (double *)ccoefs,
                     lend, xyzd[0], xyzd[1], xyzd[2], (double *)dnorms, lmnd[0], lmnd[1], lmnd[2],
                     (double *)dexps, (double *)dcoefs);
}

double ref_chgp_Fgamma(double m, double x) { return Fgamma(m, x); }
