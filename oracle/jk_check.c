/*
 * Fast FP64 CPU checker for the direct-SCF Coulomb/exchange (J/K) build.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links or calls this file;
 * the tests, the smoke check and bench.py's CPU legs use it as the checker
 * the CUDA path is compared with, and as the timed CPU baseline.
 *
 * The arithmetic is the one jk_oracle.c restates from the reference
 * (Rys quadrature with the 2D recurrences c0x/cpx/b00/b10/b01,
 * electrolites/codegen/gen_khigh.py:128-181; roots u = t^2 with weights
 * summing to F_0, electrolites/kernels/fastk_prologue.cu:69-121; prefactor
 * 2 pi^(5/2) / (p q sqrt(p+q)), fastk_prologue.cu:296-297; the screening
 * test q_ij + q_kl + max dm_cond > log(tol), fastk_prologue.cu:137-165 and
 * electrolites/kernels/fastjk_prologue.cu:26-57; the PySCF contractions
 * vj[k,l] = sum_ij (ij|kl) D[j,i], vk[i,l] = sum_jk (ij|kl) D[j,k] over the
 * distinct index permutations of each unique shell quartet), organised for
 * speed instead of for line-by-line readability:
 *   - Rys roots and weights in double from piecewise Chebyshev fits
 *     (unit intervals on [0, CHK_XMAX), degree CHK_DEG), built once per
 *     process by sampling jk_oracle.c's long-double solver (oracle_rys) at
 *     the Chebyshev nodes, and the x -> infinity limit (Hermite nodes,
 *     u x -> t_i^2, w sqrt(x) -> W_i) taken from the same solver at a large
 *     argument.  No table of the product is read;
 *   - primitive-pair data (exponent sum, centre, exp(-mu R^2) c_a c_b) built
 *     once per shell pair, with the reference's exponent cut-off
 *     (mu R^2 > 60: pair dropped);
 *   - the Cartesian (e0|f0) block accumulated over primitives and roots,
 *     then one horizontal transfer per quartet (bra, then ket);
 *   - kets visited in descending Schwarz order per bra pair, so the loop
 *     stops at the first ket that cannot pass;
 *   - OpenMP over bra shell pairs with private J/K accumulators.
 * A build can be split into S interleaved shards of bra pairs (shard s takes
 * the bra pairs of rank s, s + S, ... in the linear pair order); the shards'
 * J/K sum to the full build.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

int oracle_rys(int n, double xd, double *roots, double *weights);

#define ATM_SLOTS 6
#define PTR_COORD 1
#define BAS_SLOTS 8
#define ATOM_OF 0
#define ANG_OF 1
#define NPRIM_OF 2
#define NCTR_OF 3
#define PTR_EXP 5
#define PTR_COEFF 6

#define CHK_LMAX 3
#define CHK_NMAX 7                 /* (ff|ff): 7 roots */
#define CHK_XMAX 96                /* fits on [0, 96); the Hermite limit above */
#define CHK_DEG 13                 /* Chebyshev degree per unit interval */
#define NCART(l) (((l) + 1) * ((l) + 2) / 2)
#define PRIM_EXP_CUTOFF 60.0

/* ---------------------------------------------------------------------- */
/* Rys roots and weights                                                   */
/* ---------------------------------------------------------------------- */
/* cheb[n-1][interval][CHK_DEG+1 monomial coefficients in s][2n values] */
static double *chk_cheb[CHK_NMAX];
static double chk_inf_r[CHK_NMAX][CHK_NMAX], chk_inf_w[CHK_NMAX][CHK_NMAX];
static int chk_ready = 0;

static void chk_rys_init(void)
{
    if (chk_ready) return;
#pragma omp critical(chk_rys_init)
    {
        if (!chk_ready) {
            const int nc = CHK_DEG + 1;
            for (int n = 1; n <= CHK_NMAX; ++n) {
                double *tab = malloc(sizeof(double) * CHK_XMAX * 2 * n * nc);
#pragma omp parallel for schedule(dynamic)
                for (int it = 0; it < CHK_XMAX; ++it) {
                    double f[CHK_DEG + 1][2 * CHK_NMAX];
                    for (int k = 0; k < nc; ++k) {
                        const double s = cos(M_PI * (k + 0.5) / nc);
                        double r[CHK_NMAX], w[CHK_NMAX];
                        oracle_rys(n, it + 0.5 + 0.5 * s, r, w);
                        for (int i = 0; i < n; ++i) {
                            f[k][i] = r[i];
                            f[k][n + i] = w[i];
                        }
                    }
                    for (int v = 0; v < 2 * n; ++v)
                        for (int j = 0; j < nc; ++j) {
                            double c = 0;
                            for (int k = 0; k < nc; ++k)
                                c += f[k][v] * cos(M_PI * j * (k + 0.5) / nc);
                            tab[((size_t)it * nc + j) * 2 * n + v] = c * (j ? 2.0 : 1.0) / nc;
                        }
                }
                /* Chebyshev series -> monomials in s, in place (long double;
                 * the coefficients decay fast, so the monomial form loses
                 * little), evaluated by Estrin's scheme */
                for (int it = 0; it < CHK_XMAX; ++it)
                    for (int v = 0; v < 2 * n; ++v) {
                        long double T[CHK_DEG + 1][CHK_DEG + 1] = {{0}}, m[CHK_DEG + 1] = {0};
                        T[0][0] = 1;
                        T[1][1] = 1;
                        for (int j = 2; j <= CHK_DEG; ++j)
                            for (int k = 0; k <= j; ++k)
                                T[j][k] = (k ? 2 * T[j - 1][k - 1] : 0) - T[j - 2][k];
                        for (int j = 0; j < nc; ++j)
                            for (int k = 0; k <= j; ++k)
                                m[k] += (long double)tab[((size_t)it * nc + j) * 2 * n + v] * T[j][k];
                        for (int k = 0; k < nc; ++k) tab[((size_t)it * nc + k) * 2 * n + v] = (double)m[k];
                    }
                chk_cheb[n - 1] = tab;
                /* Hermite limit: exp(-x) corrections vanish at this argument */
                const double xb = 1.0e4;
                double r[CHK_NMAX], w[CHK_NMAX];
                oracle_rys(n, xb, r, w);
                for (int i = 0; i < n; ++i) {
                    chk_inf_r[n - 1][i] = r[i] * xb;
                    chk_inf_w[n - 1][i] = w[i] * sqrt(xb);
                }
            }
            __atomic_store_n(&chk_ready, 1, __ATOMIC_RELEASE);
        }
    }
}

static inline __attribute__((always_inline)) void chk_rys(const int n, double x,
                                                          double *r, double *w)
{
    if (x >= CHK_XMAX) {
        const double ix = 1.0 / x, sx = sqrt(ix);
        for (int i = 0; i < n; ++i) {
            r[i] = chk_inf_r[n - 1][i] * ix;
            w[i] = chk_inf_w[n - 1][i] * sx;
        }
        return;
    }
    const int it = (int)x;
    const double s = 2.0 * (x - it) - 1.0;
    const double *c = chk_cheb[n - 1] + (size_t)it * 2 * n * (CHK_DEG + 1);
    /* p(s) = sum_k a_k s^k by Estrin's scheme, all 2n values side by side */
    const double t2 = s * s, t4 = t2 * t2, t8 = t4 * t4;
    const int w2 = 2 * n;
#pragma GCC unroll 14
    for (int v = 0; v < 2 * n; ++v) {
        const double *a = c + v;
        const double p01 = fma(a[1 * w2], s, a[0]), p23 = fma(a[3 * w2], s, a[2 * w2]);
        const double p45 = fma(a[5 * w2], s, a[4 * w2]), p67 = fma(a[7 * w2], s, a[6 * w2]);
        const double p89 = fma(a[9 * w2], s, a[8 * w2]), pab = fma(a[11 * w2], s, a[10 * w2]);
        const double pcd = fma(a[13 * w2], s, a[12 * w2]);
        const double q0 = fma(p23, t2, p01), q1 = fma(p67, t2, p45), q2 = fma(pab, t2, p89);
        const double val = fma(fma(pcd, t4, q2), t8, fma(q1, t4, q0));
        if (v < n) r[v] = val; else w[v - n] = val;
    }
}

/* exported for the tests: the checker's roots and weights */
int check_rys(int n, double x, double *r, double *w)
{
    if (n < 1 || n > CHK_NMAX || !(x >= 0)) return 1;
    chk_rys_init();
    chk_rys(n, x, r, w);
    return 0;
}

/* ---------------------------------------------------------------------- */
/* Cartesian components (PySCF order) and the horizontal transfer          */
/* ---------------------------------------------------------------------- */
/* components (lx, ly, lz) of level L, PySCF order */
static const int cc[7][28][3] = {
    {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}},
    {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}},
    {{2, 0, 0}, {1, 1, 0}, {1, 0, 1}, {0, 2, 0}, {0, 1, 1}, {0, 0, 2}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}},
    {{3, 0, 0}, {2, 1, 0}, {2, 0, 1}, {1, 2, 0}, {1, 1, 1}, {1, 0, 2}, {0, 3, 0}, {0, 2, 1}, {0, 1, 2}, {0, 0, 3}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}},
    {{4, 0, 0}, {3, 1, 0}, {3, 0, 1}, {2, 2, 0}, {2, 1, 1}, {2, 0, 2}, {1, 3, 0}, {1, 2, 1}, {1, 1, 2}, {1, 0, 3}, {0, 4, 0}, {0, 3, 1}, {0, 2, 2}, {0, 1, 3}, {0, 0, 4}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}},
    {{5, 0, 0}, {4, 1, 0}, {4, 0, 1}, {3, 2, 0}, {3, 1, 1}, {3, 0, 2}, {2, 3, 0}, {2, 2, 1}, {2, 1, 2}, {2, 0, 3}, {1, 4, 0}, {1, 3, 1}, {1, 2, 2}, {1, 1, 3}, {1, 0, 4}, {0, 5, 0}, {0, 4, 1}, {0, 3, 2}, {0, 2, 3}, {0, 1, 4}, {0, 0, 5}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}},
    {{6, 0, 0}, {5, 1, 0}, {5, 0, 1}, {4, 2, 0}, {4, 1, 1}, {4, 0, 2}, {3, 3, 0}, {3, 2, 1}, {3, 1, 2}, {3, 0, 3}, {2, 4, 0}, {2, 3, 1}, {2, 2, 2}, {2, 1, 3}, {2, 0, 4}, {1, 5, 0}, {1, 4, 1}, {1, 3, 2}, {1, 2, 3}, {1, 1, 4}, {1, 0, 5}, {0, 6, 0}, {0, 5, 1}, {0, 4, 2}, {0, 3, 3}, {0, 2, 4}, {0, 1, 5}, {0, 0, 6}}};
static int cidx_tab[7][7][7]; /* (lx, ly, lz) -> index within its level */
static int comps_ready = 0;

static void comps_init(void)
{
    if (comps_ready) return;
    for (int L = 0; L <= 6; ++L) {
        int n = 0;
        for (int lx = L; lx >= 0; --lx)
            for (int ly = L - lx; ly >= 0; --ly, ++n) cidx_tab[lx][ly][L - lx - ly] = n;
    }
    comps_ready = 1;
}

/*
 * in: the components of levels l1 .. l1+l2 concatenated (PySCF order within
 * a level), read with stride `is`; out[a * NCART(l2) + b] for a at level l1
 * and b at level l2, written with stride `os`:
 *   (a, b + 1_d| = (a + 1_d, b| + R_d (a, b|
 */
static void hrr(const double *in, int is, int l1, int l2, const double R[3],
                double *out, int os)
{
    if (l2 == 0) {
        for (int a = 0; a < NCART(l1); ++a) out[a * os] = in[a * is];
        return;
    }
    /* cur[la - l1][a * nb + b] for b at level m */
    double cur[7][100], nxt[7][100];
    int off = 0;
    for (int la = l1; la <= l1 + l2; ++la) {
        for (int a = 0; a < NCART(la); ++a) cur[la - l1][a] = in[(off + a) * is];
        off += NCART(la);
    }
    for (int m = 0; m < l2; ++m) {
        const int nbo = NCART(m), nbn = NCART(m + 1);
        for (int la = l1; la <= l1 + l2 - m - 1; ++la) {
            const int na = NCART(la);
            for (int b = 0; b < nbn; ++b) {
                const int *bc = cc[m + 1][b];
                const int d = bc[0] ? 0 : (bc[1] ? 1 : 2);
                int bp[3] = {bc[0], bc[1], bc[2]};
                bp[d] -= 1;
                const int bo = cidx_tab[bp[0]][bp[1]][bp[2]];
                for (int a = 0; a < na; ++a) {
                    const int *ac = cc[la][a];
                    int ap[3] = {ac[0], ac[1], ac[2]};
                    ap[d] += 1;
                    const int a1 = cidx_tab[ap[0]][ap[1]][ap[2]];
                    nxt[la - l1][a * nbn + b] = cur[la + 1 - l1][a1 * nbo + bo] +
                                                R[d] * cur[la - l1][a * nbo + bo];
                }
            }
        }
        for (int la = l1; la <= l1 + l2 - m - 1; ++la)
            memcpy(cur[la - l1], nxt[la - l1], sizeof(double) * NCART(la) * nbn);
    }
    const int nb = NCART(l2);
    for (int a = 0; a < NCART(l1); ++a)
        for (int b = 0; b < nb; ++b) out[(a * nb + b) * os] = cur[0][a * nb + b];
}

/* ---------------------------------------------------------------------- */
/* shells and primitive pairs                                              */
/* ---------------------------------------------------------------------- */
typedef struct {
    int l, nprim, ao0, atom;
    double r[3];
    const double *exps;
    double coef[32];
} CShell;

typedef struct {
    double a, ha;              /* exponent sum a, 0.5 / a */
    double px, py, pz;         /* centre */
    double k;                  /* exp(-mu R^2) c_a c_b / a */
} PrimPair;

typedef struct {
    int ish, jsh;
    int p0, np;                /* primitive pairs [p0, p0 + np) */
    double q;                  /* log sqrt max |(ab|ab)| */
} ShellPair;

static double chk_common_fac(int l)
{
    if (l == 0) return 0.282094791773878143;   /* 1/(2 sqrt(pi)) */
    if (l == 1) return 0.488602511902919921;   /* sqrt(3/(4 pi)) */
    return 1.0;
}

typedef struct {
    int nbas, nao, npair;
    CShell *sh;
    ShellPair *pairs;          /* every i >= j, index i(i+1)/2 + j */
    PrimPair *prim;
    double omega;
} Basis;

static void basis_free(Basis *B)
{
    free(B->sh);
    free(B->pairs);
    free(B->prim);
}

static int basis_load(Basis *B, const int *atm, const int *bas, int nbas,
                      const double *env, const int *ao_loc, double omega)
{
    memset(B, 0, sizeof(*B));
    B->nbas = nbas;
    B->nao = ao_loc[nbas];
    B->omega = omega;
    B->sh = malloc(sizeof(CShell) * nbas);
    if (!B->sh) return 2;
    for (int s = 0; s < nbas; ++s) {
        const int *b = bas + s * BAS_SLOTS;
        CShell *c = B->sh + s;
        c->l = b[ANG_OF];
        c->nprim = b[NPRIM_OF];
        if (c->l < 0 || c->l > CHK_LMAX || c->nprim < 1 || c->nprim > 32 || b[NCTR_OF] != 1)
            return 1;
        c->atom = b[ATOM_OF];
        c->exps = env + b[PTR_EXP];
        const double f = chk_common_fac(c->l);
        for (int p = 0; p < c->nprim; ++p) c->coef[p] = env[b[PTR_COEFF] + p] * f;
        const double *rc = env + atm[b[ATOM_OF] * ATM_SLOTS + PTR_COORD];
        c->r[0] = rc[0];
        c->r[1] = rc[1];
        c->r[2] = rc[2];
        c->ao0 = ao_loc[s];
    }
    const long long npair = (long long)nbas * (nbas + 1) / 2;
    B->npair = (int)npair;
    B->pairs = malloc(sizeof(ShellPair) * npair);
    long long nprim = 0;
    for (int i = 0; i < nbas; ++i)
        for (int j = 0; j <= i; ++j) nprim += (long long)B->sh[i].nprim * B->sh[j].nprim;
    B->prim = malloc(sizeof(PrimPair) * (nprim ? nprim : 1));
    if (!B->pairs || !B->prim) return 2;
    long long p0 = 0;
    for (int i = 0; i < nbas; ++i)
        for (int j = 0; j <= i; ++j) {
            ShellPair *sp = B->pairs + (long long)i * (i + 1) / 2 + j;
            /* the shell of larger l first: (ij|kl) = (ji|kl), and the
             * transfer then always runs from the larger shell */
            const int swap = B->sh[j].l > B->sh[i].l;
            const int i1 = swap ? j : i, j1 = swap ? i : j;
            const CShell *a = B->sh + i1, *b = B->sh + j1;
            sp->ish = i1;
            sp->jsh = j1;
            sp->p0 = (int)p0;
            const double AB[3] = {a->r[0] - b->r[0], a->r[1] - b->r[1], a->r[2] - b->r[2]};
            const double rr = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
            int np = 0;
            for (int pa = 0; pa < a->nprim; ++pa)
                for (int pb = 0; pb < b->nprim; ++pb) {
                    const double ea = a->exps[pa], eb = b->exps[pb], s = ea + eb;
                    const double mu = ea * eb / s;
                    if (mu * rr > PRIM_EXP_CUTOFF) continue;
                    PrimPair *pp = B->prim + p0 + np;
                    pp->a = s;
                    pp->px = (ea * a->r[0] + eb * b->r[0]) / s;
                    pp->py = (ea * a->r[1] + eb * b->r[1]) / s;
                    pp->pz = (ea * a->r[2] + eb * b->r[2]) / s;
                    pp->ha = 0.5 / s;
                    pp->k = exp(-mu * rr) * a->coef[pa] * b->coef[pb] / s;
                    ++np;
                }
            sp->np = np;
            p0 += np;
        }
    return 0;
}

/* ---------------------------------------------------------------------- */
/* one shell quartet                                                       */
/* ---------------------------------------------------------------------- */
typedef struct {
    double acc[74 * 74];       /* (e0|f0), F-major: acc[f * nE + e] */
    double tb[74 * 100];       /* after the bra transfer: tb[f * nij + ij] */
} Work;

/* (e0|f0) += sum over primitive quartets and roots of the 2D-integral
 * products; LIJ, LKL are literal constants at every call site */
static inline __attribute__((always_inline)) void
prim_loop(const int LI, const int LJ, const int LK, const int LL, const PrimPair *bp, int nb,
          const PrimPair *kp, int nk, const double *A, const double *C, double om2, double *acc)
{
    const int LIJ = LI + LJ, LKL = LK + LL;
    const int NR = (LIJ + LKL) / 2 + 1;
    const int NF1 = LKL + 1;
    const double PI_FAC = 2.0 * 17.493418327624862846;   /* 2 pi^(5/2) */
    int nE = 0;
    for (int e = LI; e <= LIJ; ++e) nE += NCART(e);
    double r[CHK_NMAX], w[CHK_NMAX];
    double g[3][(LIJ + 1) * (LKL + 1)];
    for (int pp = 0; pp < nb; ++pp) {
        const PrimPair *P = bp + pp;
        const double ap = P->a;
        const double PA[3] = {P->px - A[0], P->py - A[1], P->pz - A[2]};
        for (int qq = 0; qq < nk; ++qq) {
            const PrimPair *Q = kp + qq;
            const double aq = Q->a;
            const double QC[3] = {Q->px - C[0], Q->py - C[1], Q->pz - C[2]};
            const double PQ[3] = {P->px - Q->px, P->py - Q->py, P->pz - Q->pz};
            const double is = 1.0 / (ap + aq);
            const double rho = ap * aq * is;
            double theta = 1.0, x = rho * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
            double fac = PI_FAC * P->k * Q->k * sqrt(is);
            if (om2 > 0) {
                theta = om2 / (om2 + rho);
                x *= theta;
                fac *= sqrt(theta);
            }
            chk_rys(NR, x, r, w);
            const double aqi = aq * is, api = ap * is;
            for (int n = 0; n < NR; ++n) {
                const double u = theta * r[n];
                const double b00 = 0.5 * u * is;
                const double b10 = (1 - aqi * u) * P->ha;
                const double b01 = (1 - api * u) * Q->ha;
                for (int d = 0; d < 3; ++d) {
                    const double c00 = PA[d] - aqi * u * PQ[d];
                    const double cp00 = QC[d] + api * u * PQ[d];
                    double *gd = g[d];
                    gd[0] = d == 2 ? fac * w[n] : 1.0;
                    if (LIJ > 0) gd[NF1] = c00 * gd[0];
                    for (int e = 1; e < LIJ; ++e)
                        gd[(e + 1) * NF1] = c00 * gd[e * NF1] + e * b10 * gd[(e - 1) * NF1];
                    for (int f = 0; f < LKL; ++f) {
                        gd[f + 1] = cp00 * gd[f] + (f ? f * b01 * gd[f - 1] : 0);
                        for (int e = 1; e <= LIJ; ++e)
                            gd[e * NF1 + f + 1] = cp00 * gd[e * NF1 + f] +
                                                  (f ? f * b01 * gd[e * NF1 + f - 1] : 0) +
                                                  e * b00 * gd[(e - 1) * NF1 + f];
                    }
                }
                if (LIJ + LKL == 0) {
                    acc[0] += g[2][0];
                    continue;
                }
                double *a = acc;
                for (int fl = LK; fl <= LKL; ++fl)
                    for (int fc = 0; fc < NCART(fl); ++fc, a += nE) {
                        const double *hx = g[0] + cc[fl][fc][0], *hy = g[1] + cc[fl][fc][1];
                        const double *hz = g[2] + cc[fl][fc][2];
                        int e = 0;
                        for (int el = LI; el <= LIJ; ++el)
                            for (int ec = 0; ec < NCART(el); ++ec, ++e)
                                a[e] += hx[cc[el][ec][0] * NF1] * hy[cc[el][ec][1] * NF1] *
                                        hz[cc[el][ec][2] * NF1];
                    }
            }
        }
    }
}

/* out[((a * nj + b) * nk + c) * nl + d] */
static void quartet(const Basis *B, const ShellPair *bra, const ShellPair *ket,
                    Work *W, double *out)
{
    const CShell *si = B->sh + bra->ish, *sj = B->sh + bra->jsh;
    const CShell *sk = B->sh + ket->ish, *sl = B->sh + ket->jsh;
    const int li = si->l, lj = sj->l, lk = sk->l, ll = sl->l;
    const int lij = li + lj, lkl = lk + ll;
    const int nroots = (lij + lkl) / 2 + 1;
    int nE = 0, nF = 0;
    for (int e = li; e <= lij; ++e) nE += NCART(e);
    for (int f = lk; f <= lkl; ++f) nF += NCART(f);
    double *acc = W->acc;
    memset(acc, 0, sizeof(double) * nE * nF);
    const double om2 = B->omega > 0 ? B->omega * B->omega : 0;
    const double *A = si->r, *C = sk->r;
    const PrimPair *bp = B->prim + bra->p0, *kp = B->prim + ket->p0;
    const int nb = bra->np, nk = ket->np;
    /* one instantiation of the primitive loop per class (li >= lj, lk >= ll) */
    switch (((li * 4 + lj) * 4 + lk) * 4 + ll) {
#define PL(I, J, K, L) case ((I * 4 + J) * 4 + K) * 4 + L: \
        prim_loop(I, J, K, L, bp, nb, kp, nk, A, C, om2, acc); break;
#define PLK(I, J) PL(I, J, 0, 0) PL(I, J, 1, 0) PL(I, J, 1, 1) PL(I, J, 2, 0) PL(I, J, 2, 1) \
                  PL(I, J, 2, 2) PL(I, J, 3, 0) PL(I, J, 3, 1) PL(I, J, 3, 2) PL(I, J, 3, 3)
    PLK(0, 0) PLK(1, 0) PLK(1, 1) PLK(2, 0) PLK(2, 1) PLK(2, 2) PLK(3, 0) PLK(3, 1) PLK(3, 2) PLK(3, 3)
#undef PLK
#undef PL
    default: break;
    }
    /* transfers: bra for every f column, then ket for every (ij) row */
    const double AB[3] = {si->r[0] - sj->r[0], si->r[1] - sj->r[1], si->r[2] - sj->r[2]};
    const double CD[3] = {sk->r[0] - sl->r[0], sk->r[1] - sl->r[1], sk->r[2] - sl->r[2]};
    const int nij = NCART(li) * NCART(lj), nkl = NCART(lk) * NCART(ll);
    for (int f = 0; f < nF; ++f) hrr(acc + f * nE, 1, li, lj, AB, W->tb + f * nij, 1);
    for (int ij = 0; ij < nij; ++ij) hrr(W->tb + ij, nij, lk, ll, CD, out + ij * nkl, 1);
}

/* ---------------------------------------------------------------------- */
/* J/K                                                                     */
/* ---------------------------------------------------------------------- */
typedef struct {
    int idx;
    double q;
} PairQ;

static int cmp_pairq(const void *a, const void *b)
{
    const double x = ((const PairQ *)a)->q, y = ((const PairQ *)b)->q;
    return x > y ? -1 : (x < y ? 1 : 0);
}

static void schwarz(Basis *B)
{
#pragma omp parallel
    {
        Work *W = malloc(sizeof(Work));
        double *buf = malloc(sizeof(double) * 10000);
#pragma omp for schedule(dynamic, 16)
        for (int p = 0; p < B->npair; ++p) {
            ShellPair *sp = B->pairs + p;
            if (sp->np == 0) {
                sp->q = -HUGE_VAL;
                continue;
            }
            quartet(B, sp, sp, W, buf);
            const int ni = NCART(B->sh[sp->ish].l), nj = NCART(B->sh[sp->jsh].l);
            double m = 0;
            for (int a = 0; a < ni; ++a)
                for (int b = 0; b < nj; ++b) {
                    const double v = fabs(buf[((a * nj + b) * ni + a) * nj + b]);
                    if (v > m) m = v;
                }
            sp->q = m > 0 ? log(sqrt(m)) : -HUGE_VAL;
        }
        free(W);
        free(buf);
    }
}

/*
 * Digest of one unique shell quartet (i >= j, k >= l, ij >= kl) into half
 * matrices: with v = (ab|cd) times the degeneracy factor sf (1/2 for each of
 * i == j, k == l, ij == kl), the eight index permutations of the quartet add
 *   J_h[c,d] += v Ds[a,b],  J_h[a,b] += v Ds[c,d]           (Ds = D + D^T)
 *   K_h(X)[a,d] += v X[b,c], [b,d] += v X[a,c], [a,c] += v X[b,d], [b,c] += v X[a,d]
 * and J = J_h + J_h^T, K = K_h(D) + K_h(D^T)^T.  Each block is summed over
 * the quartet before it is added to the matrices.
 */
static inline __attribute__((always_inline)) void
digest(const double *v, const int NI, const int NJ, const int NK, const int NL, size_t i0,
       size_t j0, size_t k0, size_t l0, double sf, const double *Ds, const double *D,
       const double *DT, size_t nao, double *Jh, double *Kh, double *KhT)
{
    if (Jh) {
        double dcd[NK * NL], jcd[NK * NL];
        for (int c = 0; c < NK; ++c)
            for (int d = 0; d < NL; ++d) {
                dcd[c * NL + d] = Ds[(k0 + c) * nao + l0 + d];
                jcd[c * NL + d] = 0;
            }
        for (int a = 0; a < NI; ++a)
            for (int b = 0; b < NJ; ++b) {
                const double *vv = v + (a * NJ + b) * NK * NL;
                const double x = Ds[(i0 + a) * nao + j0 + b];
                double sab = 0;
                for (int cd = 0; cd < NK * NL; ++cd) {
                    jcd[cd] += vv[cd] * x;
                    sab += vv[cd] * dcd[cd];
                }
                Jh[(i0 + a) * nao + j0 + b] += sf * sab;
            }
        for (int c = 0; c < NK; ++c)
            for (int d = 0; d < NL; ++d) Jh[(k0 + c) * nao + l0 + d] += sf * jcd[c * NL + d];
    }
    if (!Kh) return;
    for (int pass = 0; pass < (KhT ? 2 : 1); ++pass) {
        /* X = D, then X = D^T (rows of the stored transpose) */
        const double *X = pass ? DT : D;
        double *out = pass ? KhT : Kh;
        double xbc[NJ * NK], xac[NI * NK], xbd[NJ * NL], xad[NI * NL];
        double kad[NI * NL], kbd[NJ * NL], kac[NI * NK], kbc[NJ * NK];
        for (int b = 0; b < NJ; ++b)
            for (int c = 0; c < NK; ++c) {
                xbc[b * NK + c] = X[(j0 + b) * nao + k0 + c];
                kbc[b * NK + c] = 0;
            }
        for (int a = 0; a < NI; ++a)
            for (int c = 0; c < NK; ++c) {
                xac[a * NK + c] = X[(i0 + a) * nao + k0 + c];
                kac[a * NK + c] = 0;
            }
        for (int b = 0; b < NJ; ++b)
            for (int d = 0; d < NL; ++d) {
                xbd[b * NL + d] = X[(j0 + b) * nao + l0 + d];
                kbd[b * NL + d] = 0;
            }
        for (int a = 0; a < NI; ++a)
            for (int d = 0; d < NL; ++d) {
                xad[a * NL + d] = X[(i0 + a) * nao + l0 + d];
                kad[a * NL + d] = 0;
            }
        for (int a = 0; a < NI; ++a)
            for (int b = 0; b < NJ; ++b)
                for (int c = 0; c < NK; ++c) {
                    const double *vv = v + ((a * NJ + b) * NK + c) * NL;
                    const double xbc_ = xbc[b * NK + c], xac_ = xac[a * NK + c];
                    double sac = 0, sbc = 0;
                    for (int d = 0; d < NL; ++d) {
                        kad[a * NL + d] += vv[d] * xbc_;
                        kbd[b * NL + d] += vv[d] * xac_;
                        sac += vv[d] * xbd[b * NL + d];
                        sbc += vv[d] * xad[a * NL + d];
                    }
                    kac[a * NK + c] += sac;
                    kbc[b * NK + c] += sbc;
                }
        for (int a = 0; a < NI; ++a)
            for (int d = 0; d < NL; ++d) out[(i0 + a) * nao + l0 + d] += sf * kad[a * NL + d];
        for (int b = 0; b < NJ; ++b)
            for (int d = 0; d < NL; ++d) out[(j0 + b) * nao + l0 + d] += sf * kbd[b * NL + d];
        for (int a = 0; a < NI; ++a)
            for (int c = 0; c < NK; ++c) out[(i0 + a) * nao + k0 + c] += sf * kac[a * NK + c];
        for (int b = 0; b < NJ; ++b)
            for (int c = 0; c < NK; ++c) out[(j0 + b) * nao + k0 + c] += sf * kbc[b * NK + c];
    }
}

/* Per-build arguments of the digest */
typedef struct {
    int n_dm;
    size_t nao, nao2;
    const double *ds, *dm, *dmt;
    double *jh, *kh, *kht;
} DigestArgs;

/* one class (LI >= LJ, LK >= LL): block, then digest of every density */
static inline __attribute__((always_inline)) void
quartet_digest(const int LI, const int LJ, const int LK, const int LL, const Basis *B,
               const ShellPair *bra, const ShellPair *ket, Work *W, double *buf, double sf,
               const DigestArgs *G)
{
    quartet(B, bra, ket, W, buf);
    const int NI = NCART(LI), NJ = NCART(LJ), NK = NCART(LK), NL = NCART(LL);
    const size_t i0 = B->sh[bra->ish].ao0, j0 = B->sh[bra->jsh].ao0;
    const size_t k0 = B->sh[ket->ish].ao0, l0 = B->sh[ket->jsh].ao0;
    for (int d = 0; d < G->n_dm; ++d) {
        const size_t o = d * G->nao2;
        digest(buf, NI, NJ, NK, NL, i0, j0, k0, l0, sf, G->ds ? G->ds + o : NULL, G->dm + o,
               G->dmt ? G->dmt + o : NULL, G->nao, G->jh ? G->jh + o : NULL,
               G->kh ? G->kh + o : NULL, G->kht ? G->kht + o : NULL);
    }
}

static void do_quartet(const Basis *B, const ShellPair *bra, const ShellPair *ket, Work *W,
                       double *buf, double sf, const DigestArgs *G)
{
    const int li = B->sh[bra->ish].l, lj = B->sh[bra->jsh].l;
    const int lk = B->sh[ket->ish].l, ll = B->sh[ket->jsh].l;
    switch (((li * 4 + lj) * 4 + lk) * 4 + ll) {
#define QD(I, J, K, L) case ((I * 4 + J) * 4 + K) * 4 + L: \
        quartet_digest(I, J, K, L, B, bra, ket, W, buf, sf, G); break;
#define QK(I, J) QD(I, J, 0, 0) QD(I, J, 1, 0) QD(I, J, 1, 1) QD(I, J, 2, 0) QD(I, J, 2, 1) \
                 QD(I, J, 2, 2) QD(I, J, 3, 0) QD(I, J, 3, 1) QD(I, J, 3, 2) QD(I, J, 3, 3)
    QK(0, 0) QK(1, 0) QK(1, 1) QK(2, 0) QK(2, 1) QK(2, 2) QK(3, 0) QK(3, 1) QK(3, 2) QK(3, 3)
#undef QK
#undef QD
    default: break;
    }
}

static int check_impl(const int *atm, const int *bas, int nbas, const double *env,
                      const int *ao_loc, const double *dm, int n_dm, double tol,
                      int with_j, int with_k, double *vj, double *vk, int nthreads,
                      long long *nquartets, double omega, int shard, int nshard,
                      double *q_out)
{
    chk_rys_init();
    comps_init();
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    if (nshard < 1 || shard < 0 || shard >= nshard) return 3;
    Basis B;
    int err = basis_load(&B, atm, bas, nbas, env, ao_loc, omega);
    if (err) {
        basis_free(&B);
        return err;
    }
    const int nao = B.nao;
    const size_t nao2 = (size_t)nao * nao;
    schwarz(&B);
    if (q_out)
        for (int i = 0; i < nbas; ++i)
            for (int j = 0; j <= i; ++j)
                q_out[i * nbas + j] = q_out[j * nbas + i] = B.pairs[(long long)i * (i + 1) / 2 + j].q;
    const int screen = tol > 0;
    const double log_tol = screen ? log(tol) : 0;
    double *dmc = malloc(sizeof(double) * nbas * nbas);
    PairQ *order = malloc(sizeof(PairQ) * B.npair);
    if (!dmc || !order) {
        free(dmc);
        free(order);
        basis_free(&B);
        return 2;
    }
    double dmax_all = -HUGE_VAL;
#pragma omp parallel for schedule(dynamic, 8) reduction(max:dmax_all)
    for (int i = 0; i < nbas; ++i)
        for (int j = 0; j < nbas; ++j) {
            double m = 0;
            for (int d = 0; d < n_dm; ++d)
                for (int a = ao_loc[i]; a < ao_loc[i + 1]; ++a)
                    for (int b = ao_loc[j]; b < ao_loc[j + 1]; ++b) {
                        const double v1 = fabs(dm[d * nao2 + (size_t)a * nao + b]);
                        const double v2 = fabs(dm[d * nao2 + (size_t)b * nao + a]);
                        if (v1 > m) m = v1;
                        if (v2 > m) m = v2;
                    }
            dmc[i * nbas + j] = m > 0 ? log(m) : -HUGE_VAL;
            if (dmc[i * nbas + j] > dmax_all) dmax_all = dmc[i * nbas + j];
        }
    /* kets in descending Schwarz order (pairs with no primitive pair last) */
    for (int p = 0; p < B.npair; ++p) {
        order[p].idx = p;
        order[p].q = B.pairs[p].q;
    }
    qsort(order, B.npair, sizeof(PairQ), cmp_pairq);
    int nthr = 1;
#ifdef _OPENMP
    nthr = omp_get_max_threads();
#endif
    /* a symmetric density stack needs no K_h(D^T): it equals K_h(D) */
    int symmetric = 1;
    for (int d = 0; d < n_dm && symmetric; ++d)
        for (int a = 0; a < nao && symmetric; ++a)
            for (int b = 0; b < a; ++b)
                if (dm[d * nao2 + (size_t)a * nao + b] != dm[d * nao2 + (size_t)b * nao + a]) {
                    symmetric = 0;
                    break;
                }
    const size_t tot = (size_t)n_dm * nao2;
    double *ds = with_j ? malloc(sizeof(double) * tot) : NULL;
    double *vj_t = with_j ? calloc((size_t)nthr * tot, sizeof(double)) : NULL;
    double *vk_t = with_k ? calloc((size_t)nthr * tot, sizeof(double)) : NULL;
    double *vkt_t = with_k && !symmetric ? calloc((size_t)nthr * tot, sizeof(double)) : NULL;
    double *dmt = with_k && !symmetric ? malloc(sizeof(double) * tot) : NULL;
    if ((with_j && (!vj_t || !ds)) || (with_k && !vk_t) || (with_k && !symmetric && (!vkt_t || !dmt))) {
        free(ds);
        free(dmt);
        free(vj_t);
        free(vk_t);
        free(vkt_t);
        free(dmc);
        free(order);
        basis_free(&B);
        return 2;
    }
    if (ds) {
#pragma omp parallel for schedule(static)
        for (int r = 0; r < n_dm * nao; ++r) {
            const int d = r / nao, a = r % nao;
            for (int b = 0; b < nao; ++b)
                ds[d * nao2 + (size_t)a * nao + b] =
                    dm[d * nao2 + (size_t)a * nao + b] + dm[d * nao2 + (size_t)b * nao + a];
        }
    }
    if (dmt) {
#pragma omp parallel for schedule(static)
        for (int r = 0; r < n_dm * nao; ++r) {
            const int d = r / nao, a = r % nao;
            for (int b = 0; b < nao; ++b)
                dmt[d * nao2 + (size_t)a * nao + b] = dm[d * nao2 + (size_t)b * nao + a];
        }
    }
    long long count = 0;
    const int nbra = (B.npair - shard + nshard - 1) / nshard;
#pragma omp parallel reduction(+:count)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double *myj = with_j ? vj_t + (size_t)tid * n_dm * nao2 : NULL;
        double *myk = with_k ? vk_t + (size_t)tid * n_dm * nao2 : NULL;
        double *mykt = vkt_t ? vkt_t + (size_t)tid * n_dm * nao2 : NULL;
        const DigestArgs G = {n_dm, (size_t)nao, nao2, ds, dm, dmt, myj, myk, mykt};
        Work *W = malloc(sizeof(Work));
        double *buf = malloc(sizeof(double) * 10000);
#pragma omp for schedule(dynamic, 8)
        for (int t = 0; t < nbra; ++t) {
            const int pij = shard + t * nshard;
            const ShellPair *bra = B.pairs + pij;
            if (bra->np == 0) continue;
            const int i = bra->ish, j = bra->jsh;
            for (int o = 0; o < B.npair; ++o) {
                const int pkl = order[o].idx;
                if (screen && bra->q + order[o].q + dmax_all <= log_tol) break;
                if (pkl > pij) continue;
                const ShellPair *ket = B.pairs + pkl;
                if (ket->np == 0) break;
                const int k = ket->ish, l = ket->jsh;
                if (screen) {
                    double dmax = -HUGE_VAL;
                    if (with_k) {
                        const double c[4] = {dmc[i * nbas + k], dmc[i * nbas + l],
                                             dmc[j * nbas + k], dmc[j * nbas + l]};
                        for (int u = 0; u < 4; ++u) if (c[u] > dmax) dmax = c[u];
                    }
                    if (with_j) {
                        if (dmc[i * nbas + j] > dmax) dmax = dmc[i * nbas + j];
                        if (dmc[k * nbas + l] > dmax) dmax = dmc[k * nbas + l];
                    }
                    if (bra->q + ket->q + dmax <= log_tol) continue;
                }
                count++;
                const double sf = (i == j ? 0.5 : 1.0) * (k == l ? 0.5 : 1.0) * (pij == pkl ? 0.5 : 1.0);
                do_quartet(&B, bra, ket, W, buf, sf, &G);
            }
        }
        free(W);
        free(buf);
    }
    /* sum the threads' half matrices, then J = J_h + J_h^T, K = K_h(D) + K_h(D^T)^T */
#pragma omp parallel for schedule(static)
    for (size_t x = 0; x < tot; ++x) {
        double sj = 0, sk = 0, st = 0;
        for (int t = 0; t < nthr; ++t) {
            if (vj_t) sj += vj_t[(size_t)t * tot + x];
            if (vk_t) sk += vk_t[(size_t)t * tot + x];
            if (vkt_t) st += vkt_t[(size_t)t * tot + x];
        }
        if (vj_t) vj_t[x] = sj;
        if (vk_t) vk_t[x] = sk;
        if (vkt_t) vkt_t[x] = st;
    }
    const double *kt = vkt_t ? vkt_t : vk_t;
#pragma omp parallel for schedule(static)
    for (int r = 0; r < n_dm * nao; ++r) {
        const int d = r / nao, a = r % nao;
        for (int b = 0; b < nao; ++b) {
            const size_t x = d * nao2 + (size_t)a * nao + b, y = d * nao2 + (size_t)b * nao + a;
            if (vj) vj[x] = vj_t ? vj_t[x] + vj_t[y] : 0;
            if (vk) vk[x] = vk_t ? vk_t[x] + kt[y] : 0;
        }
    }
    if (nquartets) *nquartets = count;
    free(ds);
    free(dmt);
    free(vj_t);
    free(vk_t);
    free(vkt_t);
    free(dmc);
    free(order);
    basis_free(&B);
    return 0;
}

/*
 * J and K for n_dm densities dm[n_dm][nao][nao] (any symmetry) in the
 * Cartesian AO basis given by ao_loc, restricted to bra shell pairs of shard
 * `shard` of `nshard` (0 of 1: the whole build).  tol <= 0 disables
 * screening; omega > 0 gives the long-range operator erf(omega r)/r.
 * vj, vk: [n_dm][nao][nao], overwritten (either may be NULL when not
 * requested).  q_out (nbas x nbas, may be NULL) receives the Schwarz table.
 */
int check_jk(const int *atm, const int *bas, int nbas, const double *env,
             const int *ao_loc, const double *dm, int n_dm, double tol,
             int with_j, int with_k, double *vj, double *vk, int nthreads,
             long long *nquartets, double omega, int shard, int nshard, double *q_out)
{
    return check_impl(atm, bas, nbas, env, ao_loc, dm, n_dm, tol, with_j, with_k, vj, vk,
                      nthreads, nquartets, omega, shard, nshard, q_out);
}

/* (ij|kl) of four shells through the checker's quartet routine */
int check_eri_shells(const int *atm, const int *bas, int nbas, const double *env,
                     const int *ao_loc, int ish, int jsh, int ksh, int lsh, double omega,
                     double *out)
{
    chk_rys_init();
    comps_init();
    if (ish < jsh || ksh < lsh) return 3;
    Basis B;
    int err = basis_load(&B, atm, bas, nbas, env, ao_loc, omega);
    if (!err) {
        Work *W = malloc(sizeof(Work));
        double *tmp = malloc(sizeof(double) * 10000);
        const ShellPair *bra = B.pairs + (long long)ish * (ish + 1) / 2 + jsh;
        const ShellPair *ket = B.pairs + (long long)ksh * (ksh + 1) / 2 + lsh;
        quartet(&B, bra, ket, W, tmp);
        /* back to the requested shell order (a stored pair may be swapped) */
        const int n1 = NCART(B.sh[bra->ish].l), n2 = NCART(B.sh[bra->jsh].l);
        const int n3 = NCART(B.sh[ket->ish].l), n4 = NCART(B.sh[ket->jsh].l);
        const int sb = bra->ish != ish, sk = ket->ish != ksh;
        for (int a = 0; a < n1; ++a)
            for (int b = 0; b < n2; ++b)
                for (int c = 0; c < n3; ++c)
                    for (int d = 0; d < n4; ++d) {
                        const int ia = sb ? b : a, ib = sb ? a : b, ic = sk ? d : c, id = sk ? c : d;
                        const int nb = sb ? n1 : n2, nc = sk ? n4 : n3, nd = sk ? n3 : n4;
                        out[((ia * nb + ib) * nc + ic) * nd + id] = tmp[((a * n2 + b) * n3 + c) * n4 + d];
                    }
        free(tmp);
        free(W);
    }
    basis_free(&B);
    return err;
}

/* ====================================================================== */
/* Nuclear gradient of the two-electron energy                             */
/* ====================================================================== */
/*
 * E(R) = j/2 Tr[Dt J[Dt]] - k c sum_s Tr[D_s K[D_s]] for symmetric densities
 * D_s (s < n_dm), Dt = sum_s D_s, c = 1/4 for one density and 1/2 for two,
 * held fixed in the AO basis while the atoms (and their basis functions)
 * move: the quantity GPU4PySCF's _jk_energy_per_atom returns per atom, which
 * the reference replaces (electrolites/fastejk.py:276-356; its factor
 * conventions at :308-316).
 *
 * Over the distinct permutations of a unique shell quartet (ij|kl) with
 * degeneracy factor sf, E collects sum_abcd W_abcd (ab|cd) with
 *   W = sf [4 j Dt_ab Dt_cd - 4 k c sum_s (D_s,ac D_s,bd + D_s,ad D_s,bc)],
 * and the derivative of a Cartesian Gaussian on centre A,
 *   d/dA_x g_a = 2 alpha g_{a+1x} - a_x g_{a-1x},
 * turns d(ab|cd)/dA into integrals over the shell raised by one (its
 * coefficients times 2 alpha) and lowered by one.  The centres of i, j and k
 * are differentiated this way; l follows from translational invariance,
 * dD = -(dA + dB + dC).  The integrals of the raised and lowered shells
 * (up to g) come from a generic-l restatement of quartet() below.
 */
#define GL_LEV 8                   /* Cartesian levels 0..7 (g + f on one pair) */
static int gcc[GL_LEV][36][3];
static int gidx[GL_LEV][GL_LEV][GL_LEV];
static int gcomps_ready = 0;

static void gcomps_init(void)
{
    if (gcomps_ready) return;
#pragma omp critical(gcomps_init)
    {
        if (!gcomps_ready) {
            for (int L = 0; L < GL_LEV; ++L) {
                int n = 0;
                for (int lx = L; lx >= 0; --lx)
                    for (int ly = L - lx; ly >= 0; --ly, ++n) {
                        gcc[L][n][0] = lx;
                        gcc[L][n][1] = ly;
                        gcc[L][n][2] = L - lx - ly;
                        gidx[lx][ly][L - lx - ly] = n;
                    }
            }
            __atomic_store_n(&gcomps_ready, 1, __ATOMIC_RELEASE);
        }
    }
}

/* hrr() for levels up to 7 */
static void ghrr(const double *in, int is, int l1, int l2, const double R[3], double *out, int os)
{
    if (l2 == 0) {
        for (int a = 0; a < NCART(l1); ++a) out[a * os] = in[a * is];
        return;
    }
    double cur[GL_LEV][160], nxt[GL_LEV][160];
    int off = 0;
    for (int la = l1; la <= l1 + l2; ++la) {
        for (int a = 0; a < NCART(la); ++a) cur[la - l1][a] = in[(off + a) * is];
        off += NCART(la);
    }
    for (int m = 0; m < l2; ++m) {
        const int nbo = NCART(m), nbn = NCART(m + 1);
        for (int la = l1; la <= l1 + l2 - m - 1; ++la) {
            const int na = NCART(la);
            for (int b = 0; b < nbn; ++b) {
                const int *bc = gcc[m + 1][b];
                const int d = bc[0] ? 0 : (bc[1] ? 1 : 2);
                int bp[3] = {bc[0], bc[1], bc[2]};
                bp[d] -= 1;
                const int bo = gidx[bp[0]][bp[1]][bp[2]];
                for (int a = 0; a < na; ++a) {
                    const int *ac = gcc[la][a];
                    int ap[3] = {ac[0], ac[1], ac[2]};
                    ap[d] += 1;
                    const int a1 = gidx[ap[0]][ap[1]][ap[2]];
                    nxt[la - l1][a * nbn + b] = cur[la + 1 - l1][a1 * nbo + bo] +
                                                R[d] * cur[la - l1][a * nbo + bo];
                }
            }
        }
        for (int la = l1; la <= l1 + l2 - m - 1; ++la)
            memcpy(cur[la - l1], nxt[la - l1], sizeof(double) * NCART(la) * nbn);
    }
    const int nb = NCART(l2);
    for (int a = 0; a < NCART(l1); ++a)
        for (int b = 0; b < nb; ++b) out[(a * nb + b) * os] = cur[0][a * nb + b];
}

typedef struct {
    double acc[100 * 100];
    double tb[100 * 150];
    PrimPair pa[32 * 32], pb[32 * 32];
} GWork;

static int pair_prims(const CShell *a, const CShell *b, PrimPair *out)
{
    const double AB[3] = {a->r[0] - b->r[0], a->r[1] - b->r[1], a->r[2] - b->r[2]};
    const double rr = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
    int np = 0;
    for (int p = 0; p < a->nprim; ++p)
        for (int q = 0; q < b->nprim; ++q) {
            const double ea = a->exps[p], eb = b->exps[q], s = ea + eb, mu = ea * eb / s;
            if (mu * rr > PRIM_EXP_CUTOFF) continue;
            PrimPair *pp = out + np++;
            pp->a = s;
            pp->ha = 0.5 / s;
            pp->px = (ea * a->r[0] + eb * b->r[0]) / s;
            pp->py = (ea * a->r[1] + eb * b->r[1]) / s;
            pp->pz = (ea * a->r[2] + eb * b->r[2]) / s;
            pp->k = exp(-mu * rr) * a->coef[p] * b->coef[q] / s;
        }
    return np;
}

/* (ij|kl) of four shells of any l <= 4 (and l_i + l_j <= 7),
 * out[((a * nj + b) * nk + c) * nl + d] */
static void eri_generic(const CShell *si, const CShell *sj, const CShell *sk, const CShell *sl,
                        double omega, GWork *W, double *out)
{
    const int li = si->l, lj = sj->l, lk = sk->l, ll = sl->l;
    const int lij = li + lj, lkl = lk + ll;
    const int nroots = (lij + lkl) / 2 + 1;
    const int NF1 = lkl + 1;
    int nE = 0, nF = 0;
    for (int e = li; e <= lij; ++e) nE += NCART(e);
    for (int f = lk; f <= lkl; ++f) nF += NCART(f);
    double *acc = W->acc;
    memset(acc, 0, sizeof(double) * nE * nF);
    const int nb = pair_prims(si, sj, W->pa), nk = pair_prims(sk, sl, W->pb);
    const double PI_FAC = 2.0 * 17.493418327624862846;
    const double om2 = omega > 0 ? omega * omega : 0;
    double r[CHK_NMAX], w[CHK_NMAX], g[3][GL_LEV * GL_LEV];
    for (int pp = 0; pp < nb; ++pp) {
        const PrimPair *P = W->pa + pp;
        const double ap = P->a;
        const double PA[3] = {P->px - si->r[0], P->py - si->r[1], P->pz - si->r[2]};
        for (int qq = 0; qq < nk; ++qq) {
            const PrimPair *Q = W->pb + qq;
            const double aq = Q->a;
            const double QC[3] = {Q->px - sk->r[0], Q->py - sk->r[1], Q->pz - sk->r[2]};
            const double PQ[3] = {P->px - Q->px, P->py - Q->py, P->pz - Q->pz};
            const double is = 1.0 / (ap + aq);
            const double rho = ap * aq * is;
            double theta = 1.0, x = rho * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
            double fac = PI_FAC * P->k * Q->k * sqrt(is);
            if (om2 > 0) {
                theta = om2 / (om2 + rho);
                x *= theta;
                fac *= sqrt(theta);
            }
            chk_rys(nroots, x, r, w);
            const double aqi = aq * is, api = ap * is;
            for (int n = 0; n < nroots; ++n) {
                const double u = theta * r[n];
                const double b00 = 0.5 * u * is;
                const double b10 = (1 - aqi * u) * P->ha;
                const double b01 = (1 - api * u) * Q->ha;
                for (int d = 0; d < 3; ++d) {
                    const double c00 = PA[d] - aqi * u * PQ[d];
                    const double cp00 = QC[d] + api * u * PQ[d];
                    double *gd = g[d];
                    gd[0] = d == 2 ? fac * w[n] : 1.0;
                    if (lij > 0) gd[NF1] = c00 * gd[0];
                    for (int e = 1; e < lij; ++e)
                        gd[(e + 1) * NF1] = c00 * gd[e * NF1] + e * b10 * gd[(e - 1) * NF1];
                    for (int f = 0; f < lkl; ++f) {
                        gd[f + 1] = cp00 * gd[f] + (f ? f * b01 * gd[f - 1] : 0);
                        for (int e = 1; e <= lij; ++e)
                            gd[e * NF1 + f + 1] = cp00 * gd[e * NF1 + f] +
                                                  (f ? f * b01 * gd[e * NF1 + f - 1] : 0) +
                                                  e * b00 * gd[(e - 1) * NF1 + f];
                    }
                }
                double *a = acc;
                for (int fl = lk; fl <= lkl; ++fl)
                    for (int fc = 0; fc < NCART(fl); ++fc, a += nE) {
                        const int fx = gcc[fl][fc][0], fy = gcc[fl][fc][1], fz = gcc[fl][fc][2];
                        int e = 0;
                        for (int el = li; el <= lij; ++el)
                            for (int ec = 0; ec < NCART(el); ++ec, ++e)
                                a[e] += g[0][gcc[el][ec][0] * NF1 + fx] * g[1][gcc[el][ec][1] * NF1 + fy] *
                                        g[2][gcc[el][ec][2] * NF1 + fz];
                    }
            }
        }
    }
    const double AB[3] = {si->r[0] - sj->r[0], si->r[1] - sj->r[1], si->r[2] - sj->r[2]};
    const double CD[3] = {sk->r[0] - sl->r[0], sk->r[1] - sl->r[1], sk->r[2] - sl->r[2]};
    const int nij = NCART(li) * NCART(lj), nkl = NCART(lk) * NCART(ll);
    for (int f = 0; f < nF; ++f) ghrr(acc + f * nE, 1, li, lj, AB, W->tb + f * nij, 1);
    for (int ij = 0; ij < nij; ++ij) ghrr(W->tb + ij, nij, lk, ll, CD, out + ij * nkl, 1);
}

/* a shell raised (coefficients times 2 alpha) or lowered by one level */
static CShell shell_shift(const CShell *s, int up)
{
    CShell t = *s;
    t.l = s->l + (up ? 1 : -1);
    if (up)
        for (int p = 0; p < s->nprim; ++p) t.coef[p] = s->coef[p] * 2.0 * s->exps[p];
    return t;
}

/*
 * d/dR of the quartet's share of E along the centre of shell position pos
 * (0: i, 1: j, 2: k): g[x] = sum_abcd W_abcd [P(.. idx+1x ..) - n_x M(.. idx-1x ..)],
 * P and M the integrals with that shell raised and lowered.
 */
static void quartet_grad_centre(const CShell *s4[4], int pos, const double *Wt, double omega,
                                GWork *W, double *bufP, double *bufM, double g[3])
{
    const CShell *sh[4] = {s4[0], s4[1], s4[2], s4[3]};
    const int n[4] = {NCART(s4[0]->l), NCART(s4[1]->l), NCART(s4[2]->l), NCART(s4[3]->l)};
    const CShell up = shell_shift(s4[pos], 1);
    sh[pos] = &up;
    eri_generic(sh[0], sh[1], sh[2], sh[3], omega, W, bufP);
    const int lm = s4[pos]->l;
    CShell dn;
    if (lm > 0) {
        dn = shell_shift(s4[pos], 0);
        sh[pos] = &dn;
        eri_generic(sh[0], sh[1], sh[2], sh[3], omega, W, bufM);
    }
    int np[4] = {n[0], n[1], n[2], n[3]}, nm[4] = {n[0], n[1], n[2], n[3]};
    np[pos] = NCART(lm + 1);
    nm[pos] = lm > 0 ? NCART(lm - 1) : 1;
    g[0] = g[1] = g[2] = 0;
    int idx[4];
    for (idx[0] = 0; idx[0] < n[0]; ++idx[0])
        for (idx[1] = 0; idx[1] < n[1]; ++idx[1])
            for (idx[2] = 0; idx[2] < n[2]; ++idx[2])
                for (idx[3] = 0; idx[3] < n[3]; ++idx[3]) {
                    const double w = Wt[((idx[0] * n[1] + idx[1]) * n[2] + idx[2]) * n[3] + idx[3]];
                    if (w == 0) continue;
                    const int *c = gcc[lm][idx[pos]];
                    for (int x = 0; x < 3; ++x) {
                        int cu[3] = {c[0], c[1], c[2]};
                        cu[x] += 1;
                        int t[4] = {idx[0], idx[1], idx[2], idx[3]};
                        t[pos] = gidx[cu[0]][cu[1]][cu[2]];
                        double v = bufP[((t[0] * np[1] + t[1]) * np[2] + t[2]) * np[3] + t[3]];
                        if (c[x] > 0) {
                            int cd[3] = {c[0], c[1], c[2]};
                            cd[x] -= 1;
                            t[pos] = gidx[cd[0]][cd[1]][cd[2]];
                            v -= c[x] * bufM[((t[0] * nm[1] + t[1]) * nm[2] + t[2]) * nm[3] + t[3]];
                        }
                        g[x] += w * v;
                    }
                }
}

/*
 * grad[natm][3] = dE/dR of E = j/2 Tr[Dt J[Dt]] - k c sum_s Tr[D_s K[D_s]]
 * (symmetric dm[n_dm][nao][nao], n_dm 1 or 2, c = 1/4 or 1/2), quartets
 * screened as check_jk screens them (tol <= 0: none).  Returns 0 on success.
 */
int check_grad_jk(const int *atm, int natm, const int *bas, int nbas, const double *env,
                  const int *ao_loc, const double *dm, int n_dm, double tol, double j_factor,
                  double k_factor, double omega, int nthreads, double *grad,
                  long long *nquartets)
{
    chk_rys_init();
    comps_init();
    gcomps_init();
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    if (n_dm < 1 || n_dm > 2) return 3;
    Basis B;
    int err = basis_load(&B, atm, bas, nbas, env, ao_loc, 0.0);
    if (err) {
        basis_free(&B);
        return err;
    }
    for (int s = 0; s < nbas; ++s)
        if (B.sh[s].l > 3) {
            basis_free(&B);
            return 1;
        }
    const int nao = B.nao;
    const size_t nao2 = (size_t)nao * nao;
    schwarz(&B);
    const int screen = tol > 0;
    const double log_tol = screen ? log(tol) : 0;
    const double cK = n_dm == 1 ? 0.25 : 0.5;
    double *dmc = malloc(sizeof(double) * nbas * nbas);
    double *dt = malloc(sizeof(double) * nao2);
    for (size_t x = 0; x < nao2; ++x) {
        double v = 0;
        for (int d = 0; d < n_dm; ++d) v += dm[d * nao2 + x];
        dt[x] = v;
    }
    double dmax_all = -HUGE_VAL;
    for (int i = 0; i < nbas; ++i)
        for (int j = 0; j < nbas; ++j) {
            double m = 0;
            for (int d = 0; d < n_dm; ++d)
                for (int a = ao_loc[i]; a < ao_loc[i + 1]; ++a)
                    for (int b = ao_loc[j]; b < ao_loc[j + 1]; ++b) {
                        const double v1 = fabs(dm[d * nao2 + (size_t)a * nao + b]);
                        const double v2 = fabs(dm[d * nao2 + (size_t)b * nao + a]);
                        if (v1 > m) m = v1;
                        if (v2 > m) m = v2;
                    }
            dmc[i * nbas + j] = m > 0 ? log(m) : -HUGE_VAL;
            if (dmc[i * nbas + j] > dmax_all) dmax_all = dmc[i * nbas + j];
        }
    int nthr = 1;
#ifdef _OPENMP
    nthr = omp_get_max_threads();
#endif
    double *gt = calloc((size_t)nthr * natm * 3, sizeof(double));
    long long count = 0;
#pragma omp parallel reduction(+:count)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double *myg = gt + (size_t)tid * natm * 3;
        GWork *W = malloc(sizeof(GWork));
        double *Wt = malloc(sizeof(double) * 10000);
        double *bP = malloc(sizeof(double) * 15 * 1000), *bM = malloc(sizeof(double) * 6 * 1000);
#pragma omp for schedule(dynamic, 4)
        for (int pij = 0; pij < B.npair; ++pij) {
            const ShellPair *bra = B.pairs + pij;
            if (bra->np == 0) continue;
            for (int pkl = 0; pkl <= pij; ++pkl) {
                const ShellPair *ket = B.pairs + pkl;
                if (ket->np == 0) continue;
                const int i = bra->ish, j = bra->jsh, k = ket->ish, l = ket->jsh;
                if (screen) {
                    double dmax = dmc[i * nbas + j];
                    const double c[5] = {dmc[k * nbas + l], dmc[i * nbas + k], dmc[i * nbas + l],
                                         dmc[j * nbas + k], dmc[j * nbas + l]};
                    for (int u = 0; u < 5; ++u) if (c[u] > dmax) dmax = c[u];
                    if (bra->q + ket->q + dmax <= log_tol) continue;
                }
                count++;
                const CShell *s4[4] = {B.sh + i, B.sh + j, B.sh + k, B.sh + l};
                const int ni = NCART(s4[0]->l), nj = NCART(s4[1]->l);
                const int nk = NCART(s4[2]->l), nl = NCART(s4[3]->l);
                const int pi = bra->ish == bra->jsh, pk = ket->ish == ket->jsh;
                const double sf = (pi ? 0.5 : 1.0) * (pk ? 0.5 : 1.0) * (pij == pkl ? 0.5 : 1.0);
                int t = 0;
                for (int a = 0; a < ni; ++a)
                    for (int b = 0; b < nj; ++b)
                        for (int c = 0; c < nk; ++c)
                            for (int d = 0; d < nl; ++d, ++t) {
                                const size_t A_ = s4[0]->ao0 + a, B_ = s4[1]->ao0 + b;
                                const size_t C_ = s4[2]->ao0 + c, D_ = s4[3]->ao0 + d;
                                double v = 4 * j_factor * dt[A_ * nao + B_] * dt[C_ * nao + D_];
                                for (int s = 0; s < n_dm; ++s) {
                                    const double *Ds = dm + s * nao2;
                                    v -= 4 * k_factor * cK *
                                         (Ds[A_ * nao + C_] * Ds[B_ * nao + D_] +
                                          Ds[A_ * nao + D_] * Ds[B_ * nao + C_]);
                                }
                                Wt[t] = sf * v;
                            }
                double gsum[3] = {0, 0, 0};
                for (int pos = 0; pos < 3; ++pos) {
                    double g[3];
                    quartet_grad_centre(s4, pos, Wt, omega, W, bP, bM, g);
                    for (int x = 0; x < 3; ++x) {
                        myg[s4[pos]->atom * 3 + x] += g[x];
                        gsum[x] += g[x];
                    }
                }
                for (int x = 0; x < 3; ++x) myg[s4[3]->atom * 3 + x] -= gsum[x];
            }
        }
        free(W);
        free(Wt);
        free(bP);
        free(bM);
    }
    for (int a = 0; a < natm * 3; ++a) {
        double v = 0;
        for (int t = 0; t < nthr; ++t) v += gt[(size_t)t * natm * 3 + a];
        grad[a] = v;
    }
    if (nquartets) *nquartets = count;
    free(gt);
    free(dmc);
    free(dt);
    basis_free(&B);
    return 0;
}
