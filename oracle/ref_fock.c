/* Test infrastructure: a C driver around the REFERENCE's own Rys engine
 * (Src/lib/utils/crys.c, linked from the reference tree by oracle/Makefile).
 *
 * It reproduces the loop of PyQuante/Ints.py:146-167 (get2ints) without the
 * Python interpreter, and the 2J-K contraction of PyQuante/Ints.py:225-238
 * (get2JmK with the fetch_jints/fetch_kints gathers of :176-193), so the
 * reference's arithmetic can be (a) checked against and (b) timed on the
 * host cores.  The only deliberate deviation is the packed index, which is
 * computed in 64 bits: Src/cints.c:413-425 overflows a C int for nbf >= 304.
 *
 * The reference engine keeps its scratch in file-scope statics
 * (Src/lib/utils/crys.h:14-15), so parallel runs use fork()ed processes,
 * never threads.
 *
 * Basis-function table (one row per contracted function, PyQuante order):
 *   origin[3*nbf], powers[3*nbf], prim_off[nbf+1],
 *   exps/coefs/pnorms[prim_off[nbf]], norms[nbf]
 * which is exactly what CGBF.coulomb (PyQuante/CGBF.py:191-199) hands to
 * crys.contr_coulomb.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/time.h>
#include <sys/wait.h>
#include <unistd.h>

double contr_coulomb(int lena, double *aexps, double *acoefs, double *anorms,
                     double xa, double ya, double za, int la, int ma, int na,
                     int lenb, double *bexps, double *bcoefs, double *bnorms,
                     double xb, double yb, double zb, int lb, int mb, int nb,
                     int lenc, double *cexps, double *ccoefs, double *cnorms,
                     double xc, double yc, double zc, int lc, int mc, int nc,
                     int lend, double *dexps, double *dcoefs, double *dnorms,
                     double xd, double yd, double zd, int ld, int md, int nd);

typedef struct {
    int64_t nbf;
    const double *origin;
    const int64_t *powers;
    const int64_t *prim_off;
    const double *exps, *coefs, *pnorms, *norms;
} bftab;

static inline int64_t pair_index(int64_t i, int64_t j) { return i * (i + 1) / 2 + j; }

/* 64-bit twin of Src/cints.c:413-425 (same ordering). */
int64_t ref_ijkl2intindex64(int64_t i, int64_t j, int64_t k, int64_t l)
{
    int64_t t, ij, kl;
    if (i < j) { t = i; i = j; j = t; }
    if (k < l) { t = k; k = l; l = t; }
    ij = pair_index(i, j);
    kl = pair_index(k, l);
    if (ij < kl) { t = ij; ij = kl; kl = t; }
    return ij * (ij + 1) / 2 + kl;
}

/* CGBF.coulomb: a.norm*b.norm*c.norm*d.norm*crys.contr_coulomb(...) */
static double cgbf_coulomb(const bftab *t, int64_t a, int64_t b, int64_t c, int64_t d)
{
#define ARGS(f) (int)(t->prim_off[f + 1] - t->prim_off[f]), (double *)t->exps + t->prim_off[f], \
                (double *)t->coefs + t->prim_off[f], (double *)t->pnorms + t->prim_off[f],     \
                t->origin[3 * f], t->origin[3 * f + 1], t->origin[3 * f + 2],                  \
                (int)t->powers[3 * f], (int)t->powers[3 * f + 1], (int)t->powers[3 * f + 2]
    double v = contr_coulomb(ARGS(a), ARGS(b), ARGS(c), ARGS(d));
#undef ARGS
    return t->norms[a] * t->norms[b] * t->norms[c] * t->norms[d] * v;
}

/* One bra row of Ints.get2ints: all (ij|kl) with kl >= ij (Ints.py:155-164).
 * Returns the number of integrals computed; writes them if out != NULL and
 * accumulates a checksum. */
static int64_t get2ints_row(const bftab *t, int64_t i, int64_t j, double *out, double *checksum)
{
    int64_t n = t->nbf, ij = pair_index(i, j), cnt = 0;
    for (int64_t k = 0; k < n; k++)
        for (int64_t l = 0; l <= k; l++) {
            int64_t kl = pair_index(k, l);
            if (ij <= kl) {
                double v = cgbf_coulomb(t, i, j, k, l);
                if (out) out[ref_ijkl2intindex64(i, j, k, l)] = v;
                *checksum += v;
                cnt++;
            }
        }
    return cnt;
}

/* Full get2ints into out[Q], Q = P(P+1)/2, P = nbf(nbf+1)/2; nproc forked
 * workers take bra rows round-robin and write into a shared mapping.       */
int ref_get2ints(int64_t nbf, const double *origin, const int64_t *powers, const int64_t *prim_off,
                 const double *exps, const double *coefs, const double *pnorms, const double *norms,
                 double *out, int nproc)
{
    bftab t = {nbf, origin, powers, prim_off, exps, coefs, pnorms, norms};
    int64_t P = nbf * (nbf + 1) / 2, Q = P * (P + 1) / 2;
    if (nproc <= 1) {
        double cs = 0;
        for (int64_t i = 0; i < nbf; i++)
            for (int64_t j = 0; j <= i; j++) get2ints_row(&t, i, j, out, &cs);
        return 0;
    }
    double *sh = mmap(NULL, (size_t)Q * sizeof(double), PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
    if (sh == MAP_FAILED) return -1;
    for (int p = 0; p < nproc; p++) {
        pid_t pid = fork();
        if (pid < 0) return -2;
        if (pid == 0) {
            double cs = 0;
            int64_t row = 0;
            for (int64_t i = 0; i < nbf; i++)
                for (int64_t j = 0; j <= i; j++, row++)
                    if (row % nproc == p) get2ints_row(&t, i, j, sh, &cs);
            _exit(0);
        }
    }
    int st, bad = 0;
    for (int p = 0; p < nproc; p++) {
        wait(&st);
        if (!WIFEXITED(st) || WEXITSTATUS(st) != 0) bad = 1;
    }
    memcpy(out, sh, (size_t)Q * sizeof(double));
    munmap(sh, (size_t)Q * sizeof(double));
    return bad ? -3 : 0;
}

/* Ints.get2JmK (Ints.py:225-238) with the gathers of fetch_jints/fetch_kints
 * (Ints.py:176-193): G[i,j] = sum_kl (2 (ij|kl) - (ik|jl)) D[k,l], i >= j,
 * mirrored to G[j,i]. */
void ref_get2JmK(int64_t nbf, const double *ints, const double *D, double *G)
{
    for (int64_t i = 0; i < nbf; i++)
        for (int64_t j = 0; j <= i; j++) {
            double s = 0;
            for (int64_t k = 0; k < nbf; k++)
                for (int64_t l = 0; l < nbf; l++)
                    s += (2 * ints[ref_ijkl2intindex64(i, j, k, l)] - ints[ref_ijkl2intindex64(i, k, j, l)]) *
                         D[k * nbf + l];
            G[i * nbf + j] = G[j * nbf + i] = s;
        }
}

static double wall(void)
{
    struct timeval tv;
    gettimeofday(&tv, NULL);
    return tv.tv_sec + 1e-6 * tv.tv_usec;
}

/* Timed sample of the reference's integral work: the bra rows whose pair
 * index ij is in rows[0..nrows) (each row = every kl >= ij, as get2ints does),
 * spread over nproc forked workers.  Returns wall seconds; *count receives the
 * number of contracted quartets evaluated. */
double ref_time_rows(int64_t nbf, const double *origin, const int64_t *powers, const int64_t *prim_off,
                     const double *exps, const double *coefs, const double *pnorms, const double *norms,
                     const int64_t *rows, int64_t nrows, int nproc, int64_t *count, double *checksum)
{
    bftab t = {nbf, origin, powers, prim_off, exps, coefs, pnorms, norms};
    int64_t *ii = malloc(nrows * sizeof(int64_t)), *jj = malloc(nrows * sizeof(int64_t));
    int64_t total = 0;
    for (int64_t r = 0; r < nrows; r++) {
        int64_t ij = rows[r], i = 0;
        while (pair_index(i + 1, 0) <= ij) i++;
        ii[r] = i;
        jj[r] = ij - pair_index(i, 0);
        total += nbf * (nbf + 1) / 2 - ij;
    }
    if (nproc < 1) nproc = 1;
    double *sh = mmap(NULL, 64 * sizeof(double) * (nproc + 1), PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
    double t0 = wall();
    for (int p = 0; p < nproc; p++) {
        pid_t pid = fork();
        if (pid == 0) {
            double cs = 0;
            for (int64_t r = p; r < nrows; r += nproc) get2ints_row(&t, ii[r], jj[r], NULL, &cs);
            sh[64 * p] = cs;
            _exit(0);
        }
    }
    int st;
    for (int p = 0; p < nproc; p++) wait(&st);
    double dt = wall() - t0;
    double cs = 0;
    for (int p = 0; p < nproc; p++) cs += sh[64 * p];
    munmap(sh, 64 * sizeof(double) * (nproc + 1));
    free(ii);
    free(jj);
    *count = total;
    *checksum = cs;
    return dt;
}

#ifdef REF_FOCK_MAIN
/* Standalone timed CPU baseline.  usage: ref_fock <basis.bin> <rows.bin> <nproc>
 * basis.bin: int64 nbf, int64 nprim, double origin[3nbf], int64 powers[3nbf],
 *            int64 prim_off[nbf+1], double exps/coefs/pnorms[nprim], norms[nbf]
 * rows.bin : int64 pair indices.  Prints one JSON object. */
static void *slurp(const char *path, size_t *len)
{
    FILE *f = fopen(path, "rb");
    if (!f) return NULL;
    fseek(f, 0, SEEK_END);
    *len = ftell(f);
    fseek(f, 0, SEEK_SET);
    void *b = malloc(*len);
    if (fread(b, 1, *len, f) != *len) { fclose(f); free(b); return NULL; }
    fclose(f);
    return b;
}

int main(int argc, char **argv)
{
    if (argc < 4) { fprintf(stderr, "usage: %s basis.bin rows.bin nproc\n", argv[0]); return 2; }
    size_t bl, rl;
    char *b = slurp(argv[1], &bl);
    int64_t *rows = slurp(argv[2], &rl);
    if (!b || !rows) { fprintf(stderr, "cannot read inputs\n"); return 2; }
    int nproc = atoi(argv[3]);
    int64_t nbf = ((int64_t *)b)[0], nprim = ((int64_t *)b)[1];
    char *p = b + 16;
    const double *origin = (const double *)p; p += 3 * nbf * 8;
    const int64_t *powers = (const int64_t *)p; p += 3 * nbf * 8;
    const int64_t *prim_off = (const int64_t *)p; p += (nbf + 1) * 8;
    const double *exps = (const double *)p; p += nprim * 8;
    const double *coefs = (const double *)p; p += nprim * 8;
    const double *pnorms = (const double *)p; p += nprim * 8;
    const double *norms = (const double *)p;
    int64_t cnt = 0;
    double cs = 0;
    double dt = ref_time_rows(nbf, origin, powers, prim_off, exps, coefs, pnorms, norms, rows,
                              (int64_t)(rl / 8), nproc, &cnt, &cs);
    printf("{\"seconds\": %.6f, \"quartets\": %lld, \"nproc\": %d, \"checksum\": %.17g}\n", dt,
           (long long)cnt, nproc, cs);
    return 0;
}
#endif
