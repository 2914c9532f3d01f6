/* Test-infrastructure shim: compiles the reference's Src/cints.c (THO engine,
 * one-electron integrals, Boys function, 32-bit ijkl2intindex) unmodified,
 * from the reference tree, and exports plain-C entry points for ctypes.
 * The CPython module-init call (Src/cints.c:973) is neutralised.            */
#define Py_InitModule(n, m) ((void *)0)
#include "Src/cints.c"

double ref_cints_coulomb_repulsion(double xa, double ya, double za, double norma, int la, int ma, int na, double alphaa,
                                   double xb, double yb, double zb, double normb, int lb, int mb, int nb, double alphab,
                                   double xc, double yc, double zc, double normc, int lc, int mc, int nc, double alphac,
                                   double xd, double yd, double zd, double normd, int ld, int md, int nd, double alphad)
{
    return coulomb_repulsion(xa, ya, za, norma, la, ma, na, alphaa, xb, yb, zb, normb, lb, mb, nb, alphab,
                             xc, yc, zc, normc, lc, mc, nc, alphac, xd, yd, zd, normd, ld, md, nd, alphad);
}

double ref_cints_overlap(double a1, int l1, int m1, int n1, double xa, double ya, double za,
                         double a2, int l2, int m2, int n2, double xb, double yb, double zb)
{
    return overlap(a1, l1, m1, n1, xa, ya, za, a2, l2, m2, n2, xb, yb, zb);
}

double ref_cints_kinetic(double a1, int l1, int m1, int n1, double xa, double ya, double za,
                         double a2, int l2, int m2, int n2, double xb, double yb, double zb)
{
    return kinetic(a1, l1, m1, n1, xa, ya, za, a2, l2, m2, n2, xb, yb, zb);
}

double ref_cints_nuclear(double x1, double y1, double z1, double norm1, int l1, int m1, int n1, double alpha1,
                         double x2, double y2, double z2, double norm2, int l2, int m2, int n2, double alpha2,
                         double x3, double y3, double z3)
{
    return nuclear_attraction(x1, y1, z1, norm1, l1, m1, n1, alpha1, x2, y2, z2, norm2, l2, m2, n2, alpha2,
                              x3, y3, z3);
}

int ref_cints_ijkl2intindex(int i, int j, int k, int l) { return ijkl2intindex(i, j, k, l); }
double ref_cints_Fgamma(double m, double x) { return Fgamma(m, x); }
int ref_cints_fact2(int n) { return fact2(n); }
