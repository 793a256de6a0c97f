/*
 * CPU oracle for the direct-SCF Coulomb/exchange (J/K) build.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links or calls this file;
 * the tests, the smoke check and the CPU-baseline leg of bench.py use it as
 * the checker the CUDA path is compared with.
 *
 * It restates, in plain C with long-double Rys roots, the arithmetic of the
 * reference J/K build:
 *   - Rys quadrature per primitive quartet with the 2D recurrences
 *     c0x/cpx/b00/b10/b01, VRR on centres i and k, then HRR i->j and k->l
 *     per root (electrolites/codegen/gen_khigh.py:128-181, and the generated
 *     kernels, e.g. electrolites/kernels/fastk_generated.cu:285-330);
 *   - roots u = t^2 and weights that sum to F_0(x)
 *     (electrolites/kernels/fastk_prologue.cu:69-121), computed here from
 *     scratch: discretised Stieltjes on exp(-x t^2) dt, Jacobi matrix
 *     eigenvalues by Sturm bisection, Christoffel weights;
 *   - the prefactor 2 pi^(5/2) / (p q sqrt(p+q)) (PI_FAC,
 *     fastk_prologue.cu:35, :296-297);
 *   - Schwarz plus density screening: keep a unique quartet when
 *     q_ij + q_kl + max(dm_cond of the blocks the build reads) > log(tol)
 *     (fastk_prologue.cu:137-165 for K; electrolites/kernels/
 *     fastjk_prologue.cu:26-57 for J and K together);
 *   - the PySCF contraction conventions vj[k,l] = sum_ij (ij|kl) D[j,i] and
 *     vk[i,l] = sum_jk (ij|kl) D[j,k], applied here to all eight index
 *     permutations of each unique quartet, written out one by one instead of
 *     the half-matrix-plus-transpose scheme the kernels use
 *     (electrolites/fastjk.py:346-357), so the two schemes check each other.
 *
 * Basis conventions follow PySCF's _atm/_bas/_env arrays: the coefficients
 * stored at PTR_COEFF already carry the radial normalisation, and libcint's
 * extra angular factor for s and p shells (1/(2 sqrt(pi)), sqrt(3/(4 pi))) is
 * applied per shell.  Cartesian components are ordered xx..., xy..., the
 * PySCF order (gen_khigh.py:64-75).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ATM_SLOTS 6
#define PTR_COORD 1
#define BAS_SLOTS 8
#define ATOM_OF 0
#define ANG_OF 1
#define NPRIM_OF 2
#define NCTR_OF 3
#define PTR_EXP 5
#define PTR_COEFF 6

#define LMAX 3
#define NROOT_MAX 7
#define NCART(l) (((l) + 1) * ((l) + 2) / 2)

typedef long double ldbl;

/* ---------------------------------------------------------------------- */
/* Gauss-Legendre rule in long double (Newton on P_m)                      */
/* ---------------------------------------------------------------------- */
#define GL_M 24
static ldbl gl_x[GL_M], gl_w[GL_M];
static int gl_ready = 0;

static void gl_init(void)
{
    if (gl_ready) return;
    for (int i = 0; i < GL_M; ++i) {
        ldbl x = cosl(3.14159265358979323846264338327950288L * (i + 0.75L) /
                      (GL_M + 0.5L));
        ldbl p0 = 1, p1 = x, dp = 0;
        for (int it = 0; it < 100; ++it) {
            p0 = 1; p1 = x;
            for (int k = 2; k <= GL_M; ++k) {
                ldbl p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
                p0 = p1; p1 = p2;
            }
            dp = GL_M * (x * p1 - p0) / (x * x - 1);
            ldbl dx = p1 / dp;
            x -= dx;
            if (fabsl(dx) < 1e-21L) break;
        }
        p0 = 1; p1 = x;
        for (int k = 2; k <= GL_M; ++k) {
            ldbl p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
            p0 = p1; p1 = p2;
        }
        dp = GL_M * (x * p1 - p0) / (x * x - 1);
        gl_x[i] = x;
        gl_w[i] = 2 / ((1 - x * x) * dp * dp);
    }
    gl_ready = 1;
}

/* ---------------------------------------------------------------------- */
/* Rys roots (u = t^2) and weights for weight exp(-x t^2) on t in [0, 1]    */
/* ---------------------------------------------------------------------- */
int oracle_rys(int n, double xd, double *roots, double *weights)
{
    if (n < 1 || n > NROOT_MAX + 2) return 1;
    gl_init();
    ldbl x = xd;
    /* composite Gauss-Legendre panels in t, finer for large x */
    ldbl width = 1.0L;
    if (x > 1) width = 8.0L / sqrtl(x);
    if (width > 1) width = 1;
    width *= 0.25L;
    int npanel = (int)ceill(1.0L / width);
    if (npanel > 64) npanel = 64;
    ldbl u[64 * GL_M], w[64 * GL_M], p[64 * GL_M], pm[64 * GL_M];
    int nn = 0;
    for (int pnl = 0; pnl < npanel; ++pnl) {
        ldbl a = pnl * width, b = a + width;
        if (pnl == npanel - 1 || b > 1) b = 1;
        for (int g = 0; g < GL_M; ++g, ++nn) {
            ldbl t = (a + b) / 2 + (b - a) / 2 * gl_x[g];
            w[nn] = (b - a) / 2 * gl_w[g] * expl(-x * t * t);
            u[nn] = t * t;
            p[nn] = 1;
            pm[nn] = 0;
        }
    }
    ldbl alpha[NROOT_MAX + 2], beta[NROOT_MAX + 2];
    /* discretised Stieltjes procedure: p holds p_j, pm holds p_{j-1} */
    ldbl norm_prev = 1;
    for (int j = 0; j < n; ++j) {
        ldbl s0 = 0, s1 = 0;
        for (int k = 0; k < nn; ++k) {
            ldbl wp = w[k] * p[k] * p[k];
            s0 += wp;
            s1 += wp * u[k];
        }
        alpha[j] = s1 / s0;
        beta[j] = (j == 0) ? s0 : s0 / norm_prev;
        norm_prev = s0;
        for (int k = 0; k < nn; ++k) {
            ldbl pn = (u[k] - alpha[j]) * p[k] - (j ? beta[j] : 0) * pm[k];
            pm[k] = p[k];
            p[k] = pn;
        }
    }
    /* eigenvalues of the Jacobi matrix by Sturm-sequence bisection */
    for (int k = 0; k < n; ++k) {
        ldbl lo = 0, hi = 1;
        for (int it = 0; it < 200; ++it) {
            ldbl mid = (lo + hi) / 2;
            if (mid == lo || mid == hi) break;
            int count = 0;
            ldbl d = alpha[0] - mid;
            if (d < 0) count++;
            for (int j = 1; j < n; ++j) {
                if (d == 0) d = 1e-4000L;
                d = (alpha[j] - mid) - beta[j] / d;
                if (d < 0) count++;
            }
            if (count > k) hi = mid; else lo = mid;
        }
        ldbl r = (lo + hi) / 2;
        /* Christoffel number with the orthonormal polynomials */
        ldbl s = 0, qm = 0, q = 1, nrm = beta[0];
        for (int j = 0; j < n; ++j) {
            s += q * q / nrm;
            if (j + 1 < n) {
                ldbl qn = (r - alpha[j]) * q - (j ? beta[j] : 0) * qm;
                qm = q; q = qn;
                nrm *= beta[j + 1];
            }
        }
        roots[k] = (double)r;
        weights[k] = (double)(1 / s);
    }
    return 0;
}

/* ---------------------------------------------------------------------- */
/* shells                                                                  */
/* ---------------------------------------------------------------------- */
typedef struct {
    int l, nprim;
    const double *exps;
    double coef[32];
    double r[3];
} Shell;

static double common_fac(int l)
{
    if (l == 0) return 0.282094791773878143;   /* 1/(2 sqrt(pi)) */
    if (l == 1) return 0.488602511902919921;   /* sqrt(3/(4 pi)) */
    return 1.0;
}

static int load_shell(Shell *s, const int *atm, const int *bas,
                      const double *env, int ish)
{
    const int *b = bas + ish * BAS_SLOTS;
    s->l = b[ANG_OF];
    s->nprim = b[NPRIM_OF];
    if (s->l < 0 || s->l > LMAX || s->nprim < 1 || s->nprim > 32 ||
        b[NCTR_OF] != 1) return 1;
    s->exps = env + b[PTR_EXP];
    double f = common_fac(s->l);
    for (int p = 0; p < s->nprim; ++p) s->coef[p] = env[b[PTR_COEFF] + p] * f;
    const double *rc = env + atm[b[ATOM_OF] * ATM_SLOTS + PTR_COORD];
    s->r[0] = rc[0]; s->r[1] = rc[1]; s->r[2] = rc[2];
    return 0;
}

/* Cartesian component list of level l in PySCF order */
static void cart_comps(int l, int (*c)[3])
{
    int n = 0;
    for (int lx = l; lx >= 0; --lx)
        for (int ly = l - lx; ly >= 0; --ly) {
            c[n][0] = lx; c[n][1] = ly; c[n][2] = l - lx - ly; ++n;
        }
}

#define PRIM_EXP_CUTOFF 60.0   /* drop a primitive pair if exp(-mu R^2) < e^-60 */

/*
 * (ij|kl) for one shell quartet, out[a][b][c][d] in Cartesian components.
 * omega > 0: the long-range operator erf(omega r)/r instead of 1/r.  Its
 * Rys quadrature is the Coulomb one on the shortened t range
 * [0, sqrt(theta)], theta = omega^2 / (omega^2 + rho): the roots and weights
 * at theta x, with the roots (t^2) scaled by theta and the weights by
 * sqrt(theta) (the reference folds the same change into one fma on
 * rsqrt(p + q), electrolites/kernels/fastk_prologue.cu:281-288).
 */
static void eri_shell_quartet(const Shell *si, const Shell *sj,
                              const Shell *sk, const Shell *sl, double omega, double *out)
{
    const int li = si->l, lj = sj->l, lk = sk->l, ll = sl->l;
    const int lij = li + lj, lkl = lk + ll;
    const int nroots = (lij + lkl) / 2 + 1;
    const int ni = NCART(li), nj = NCART(lj), nk = NCART(lk), nl = NCART(ll);
    int ci[10][3], cj[10][3], ck[10][3], cl[10][3];
    cart_comps(li, ci); cart_comps(lj, cj); cart_comps(lk, ck); cart_comps(ll, cl);
    const int nout = ni * nj * nk * nl;
    for (int n = 0; n < nout; ++n) out[n] = 0;

    double AB[3], CD[3];
    for (int d = 0; d < 3; ++d) {
        AB[d] = si->r[d] - sj->r[d];
        CD[d] = sk->r[d] - sl->r[d];
    }
    const double rr_ab = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
    const double rr_cd = CD[0] * CD[0] + CD[1] * CD[1] + CD[2] * CD[2];
    const double PI_FAC = 2.0 * pow(M_PI, 2.5);

    /* 2D integrals: G[dim][e][f] and the transferred I[dim][a][b][c][d] */
    double G[3][7][7];
    double Ib[3][4][4][7];          /* after bra HRR: [a][b][f] */
    double I[3][4][4][4][4];
    double roots[NROOT_MAX], weights[NROOT_MAX];

    for (int pi = 0; pi < si->nprim; ++pi)
    for (int pj = 0; pj < sj->nprim; ++pj) {
        const double ai = si->exps[pi], aj = sj->exps[pj];
        const double p = ai + aj;
        const double mu_ab = ai * aj / p;
        if (mu_ab * rr_ab > PRIM_EXP_CUTOFF) continue;
        const double kab = exp(-mu_ab * rr_ab) * si->coef[pi] * sj->coef[pj];
        double P[3];
        for (int d = 0; d < 3; ++d) P[d] = (ai * si->r[d] + aj * sj->r[d]) / p;
        for (int pk = 0; pk < sk->nprim; ++pk)
        for (int pl = 0; pl < sl->nprim; ++pl) {
            const double ak = sk->exps[pk], al = sl->exps[pl];
            const double q = ak + al;
            const double mu_cd = ak * al / q;
            if (mu_cd * rr_cd > PRIM_EXP_CUTOFF) continue;
            const double kcd = exp(-mu_cd * rr_cd) * sk->coef[pk] * sl->coef[pl];
            double Q[3], PQ[3];
            for (int d = 0; d < 3; ++d) {
                Q[d] = (ak * sk->r[d] + al * sl->r[d]) / q;
                PQ[d] = P[d] - Q[d];
            }
            const double s = p + q;
            const double rho = p * q / s;
            const double theta = omega > 0 ? omega * omega / (omega * omega + rho) : 1.0;
            const double x = theta * rho * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
            const double fac = PI_FAC / (p * q * sqrt(s)) * kab * kcd * sqrt(theta);
            oracle_rys(nroots, x, roots, weights);
            for (int r = 0; r < nroots; ++r) {
                const double u = theta * roots[r];
                const double b00 = 0.5 * u / s;
                const double b10 = (1 - q / s * u) / (2 * p);
                const double b01 = (1 - p / s * u) / (2 * q);
                for (int d = 0; d < 3; ++d) {
                    const double c00 = (P[d] - si->r[d]) - q / s * u * PQ[d];
                    const double cp00 = (Q[d] - sk->r[d]) + p / s * u * PQ[d];
                    double (*g)[7] = G[d];
                    g[0][0] = (d == 2) ? fac * weights[r] : 1.0;
                    for (int e = 0; e < lij; ++e)
                        g[e + 1][0] = c00 * g[e][0] + (e ? e * b10 * g[e - 1][0] : 0);
                    for (int f = 0; f < lkl; ++f)
                        for (int e = 0; e <= lij; ++e)
                            g[e][f + 1] = cp00 * g[e][f]
                                        + (f ? f * b01 * g[e][f - 1] : 0)
                                        + (e ? e * b00 * g[e - 1][f] : 0);
                    /* bra HRR: (a, b+1| = (a+1, b| + AB (a, b| */
                    for (int f = 0; f <= lkl; ++f) {
                        double t[7][4];
                        for (int e = 0; e <= lij; ++e) t[e][0] = g[e][f];
                        for (int b = 1; b <= lj; ++b)
                            for (int a = 0; a <= lij - b; ++a)
                                t[a][b] = t[a + 1][b - 1] + AB[d] * t[a][b - 1];
                        for (int a = 0; a <= li; ++a)
                            for (int b = 0; b <= lj; ++b) Ib[d][a][b][f] = t[a][b];
                    }
                    /* ket HRR: |c, d+1) = |c+1, d) + CD |c, d) */
                    for (int a = 0; a <= li; ++a)
                    for (int b = 0; b <= lj; ++b) {
                        double t[7][4];
                        for (int f = 0; f <= lkl; ++f) t[f][0] = Ib[d][a][b][f];
                        for (int dd = 1; dd <= ll; ++dd)
                            for (int c = 0; c <= lkl - dd; ++c)
                                t[c][dd] = t[c + 1][dd - 1] + CD[d] * t[c][dd - 1];
                        for (int c = 0; c <= lk; ++c)
                            for (int dd = 0; dd <= ll; ++dd)
                                I[d][a][b][c][dd] = t[c][dd];
                    }
                }
                int n = 0;
                for (int a = 0; a < ni; ++a)
                for (int b = 0; b < nj; ++b)
                for (int c = 0; c < nk; ++c)
                for (int e = 0; e < nl; ++e, ++n) {
                    out[n] += I[0][ci[a][0]][cj[b][0]][ck[c][0]][cl[e][0]]
                            * I[1][ci[a][1]][cj[b][1]][ck[c][1]][cl[e][1]]
                            * I[2][ci[a][2]][cj[b][2]][ck[c][2]][cl[e][2]];
                }
            }
        }
    }
}

int oracle_eri_shells_rs(const int *atm, const int *bas, const double *env,
                         int ish, int jsh, int ksh, int lsh, double omega, double *out)
{
    Shell s[4];
    gl_init();
    if (load_shell(&s[0], atm, bas, env, ish) || load_shell(&s[1], atm, bas, env, jsh) ||
        load_shell(&s[2], atm, bas, env, ksh) || load_shell(&s[3], atm, bas, env, lsh))
        return 1;
    eri_shell_quartet(&s[0], &s[1], &s[2], &s[3], omega, out);
    return 0;
}

int oracle_eri_shells(const int *atm, const int *bas, const double *env,
                      int ish, int jsh, int ksh, int lsh, double *out)
{
    return oracle_eri_shells_rs(atm, bas, env, ish, jsh, ksh, lsh, 0.0, out);
}

/* q_cond[ish*nbas+jsh] = log(sqrt(max_ab |(ab|ab)|)) for every shell pair */
int oracle_q_cond(const int *atm, const int *bas, int nbas, const double *env,
                  double *q_cond)
{
    gl_init();
    int err = 0;
#pragma omp parallel for schedule(dynamic) reduction(|:err)
    for (int ish = 0; ish < nbas; ++ish) {
        double buf[10 * 10 * 10 * 10];
        Shell si, sj;
        if (load_shell(&si, atm, bas, env, ish)) { err |= 1; continue; }
        for (int jsh = 0; jsh <= ish; ++jsh) {
            if (load_shell(&sj, atm, bas, env, jsh)) { err |= 1; continue; }
            eri_shell_quartet(&si, &sj, &si, &sj, 0.0, buf);
            int ni = NCART(si.l), nj = NCART(sj.l);
            double m = 0;
            for (int a = 0; a < ni; ++a)
                for (int b = 0; b < nj; ++b) {
                    double v = fabs(buf[((a * nj + b) * ni + a) * nj + b]);
                    if (v > m) m = v;
                }
            double q = (m > 0) ? log(sqrt(m)) : -HUGE_VAL;
            q_cond[ish * nbas + jsh] = q;
            q_cond[jsh * nbas + ish] = q;
        }
    }
    return err;
}

/*
 * J and K for n_dm densities dm[n_dm][nao][nao] (any symmetry) in the
 * Cartesian AO basis given by ao_loc.  tol <= 0 disables screening.
 * vj, vk: [n_dm][nao][nao], overwritten.  Returns the number of unique shell
 * quartets evaluated through *nquartets when it is not NULL.
 */
static int jk_impl(const int *atm, const int *bas, int nbas, const double *env,
                   const int *ao_loc, const double *dm, int n_dm, double tol,
                   int with_j, int with_k, double *vj, double *vk, int nthreads,
                   long long *nquartets, const long long *ij_list, long long n_list,
                   double omega)
{
    gl_init();
    const int nao = ao_loc[nbas];
    const size_t nao2 = (size_t)nao * nao;
    Shell *sh = malloc(sizeof(Shell) * nbas);
    double *q = malloc(sizeof(double) * nbas * nbas);
    double *dmc = malloc(sizeof(double) * nbas * nbas);
    if (!sh || !q || !dmc) { free(sh); free(q); free(dmc); return 2; }
    for (int i = 0; i < nbas; ++i)
        if (load_shell(&sh[i], atm, bas, env, i)) {
            free(sh); free(q); free(dmc); return 1;
        }
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    int screen = tol > 0;
    if (screen) {
        oracle_q_cond(atm, bas, nbas, env, q);
        for (int i = 0; i < nbas; ++i)
            for (int j = 0; j < nbas; ++j) {
                double m = 0;
                for (int d = 0; d < n_dm; ++d)
                    for (int a = ao_loc[i]; a < ao_loc[i + 1]; ++a)
                        for (int b = ao_loc[j]; b < ao_loc[j + 1]; ++b) {
                            double v1 = fabs(dm[d * nao2 + (size_t)a * nao + b]);
                            double v2 = fabs(dm[d * nao2 + (size_t)b * nao + a]);
                            if (v1 > m) m = v1;
                            if (v2 > m) m = v2;
                        }
                dmc[i * nbas + j] = (m > 0) ? log(m) : -HUGE_VAL;
            }
    }
    const double log_tol = screen ? log(tol) : 0;
    const long long npair = (long long)nbas * (nbas + 1) / 2;
    int nthr = 1;
#ifdef _OPENMP
    nthr = omp_get_max_threads();
#endif
    double *vj_t = calloc((size_t)nthr * n_dm * nao2, sizeof(double));
    double *vk_t = calloc((size_t)nthr * n_dm * nao2, sizeof(double));
    if (!vj_t || !vk_t) { free(sh); free(q); free(dmc); free(vj_t); free(vk_t); return 2; }
    long long count = 0;
    const long long ntask = ij_list ? n_list : npair;

#pragma omp parallel reduction(+:count)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double *myj = vj_t + (size_t)tid * n_dm * nao2;
        double *myk = vk_t + (size_t)tid * n_dm * nao2;
        double *buf = malloc(sizeof(double) * 10000);
#pragma omp for schedule(dynamic, 4)
        for (long long task = 0; task < ntask; ++task) {
            const long long ij = ij_list ? ij_list[task] : task;
            if (ij < 0 || ij >= npair) continue;
            int i = (int)((sqrt(8.0 * ij + 1) - 1) / 2);
            while ((long long)i * (i + 1) / 2 > ij) --i;
            while ((long long)(i + 1) * (i + 2) / 2 <= ij) ++i;
            int j = (int)(ij - (long long)i * (i + 1) / 2);
            for (long long kl = 0; kl <= ij; ++kl) {
                int k = (int)((sqrt(8.0 * kl + 1) - 1) / 2);
                while ((long long)k * (k + 1) / 2 > kl) --k;
                while ((long long)(k + 1) * (k + 2) / 2 <= kl) ++k;
                int l = (int)(kl - (long long)k * (k + 1) / 2);
                if (screen) {
                    double dmax = -HUGE_VAL;
                    if (with_k) {
                        double c[4] = {dmc[i * nbas + k], dmc[i * nbas + l],
                                       dmc[j * nbas + k], dmc[j * nbas + l]};
                        for (int t = 0; t < 4; ++t) if (c[t] > dmax) dmax = c[t];
                    }
                    if (with_j) {
                        if (dmc[i * nbas + j] > dmax) dmax = dmc[i * nbas + j];
                        if (dmc[k * nbas + l] > dmax) dmax = dmc[k * nbas + l];
                    }
                    if (q[i * nbas + j] + q[k * nbas + l] + dmax <= log_tol) continue;
                }
                count++;
                eri_shell_quartet(&sh[i], &sh[j], &sh[k], &sh[l], omega, buf);
                const int ni = NCART(sh[i].l), nj = NCART(sh[j].l);
                const int nk = NCART(sh[k].l), nl = NCART(sh[l].l);
                const int i0 = ao_loc[i], j0 = ao_loc[j], k0 = ao_loc[k], l0 = ao_loc[l];
                /* the distinct index permutations of this shell quartet */
                int perms[8][4] = {{0,1,2,3},{1,0,2,3},{0,1,3,2},{1,0,3,2},
                                   {2,3,0,1},{3,2,0,1},{2,3,1,0},{3,2,1,0}};
                int seen[8] = {0};
                int shl[4] = {i, j, k, l};
                for (int p = 0; p < 8; ++p) {
                    for (int p2 = 0; p2 < p; ++p2) {
                        if (seen[p2] && shl[perms[p2][0]] == shl[perms[p][0]] &&
                            shl[perms[p2][1]] == shl[perms[p][1]] &&
                            shl[perms[p2][2]] == shl[perms[p][2]] &&
                            shl[perms[p2][3]] == shl[perms[p][3]]) goto skip;
                    }
                    seen[p] = 1;
                    {
                        int loc[4] = {i0, j0, k0, l0};
                        int n[4] = {ni, nj, nk, nl};
                        const int *pm = perms[p];
                        int A = pm[0], B = pm[1], C = pm[2], D = pm[3];
                        int idx[4];
                        for (idx[0] = 0; idx[0] < ni; ++idx[0])
                        for (idx[1] = 0; idx[1] < nj; ++idx[1])
                        for (idx[2] = 0; idx[2] < nk; ++idx[2])
                        for (idx[3] = 0; idx[3] < nl; ++idx[3]) {
                            double v = buf[((idx[0] * nj + idx[1]) * nk + idx[2]) * nl + idx[3]];
                            if (v == 0) continue;
                            size_t a = loc[A] + idx[A], b = loc[B] + idx[B];
                            size_t c = loc[C] + idx[C], e = loc[D] + idx[D];
                            for (int d = 0; d < n_dm; ++d) {
                                const double *D_ = dm + d * nao2;
                                /* (ab|ce): vj[c,e] += v D[b,a]; vk[a,e] += v D[b,c] */
                                if (with_j) myj[d * nao2 + c * nao + e] += v * D_[b * nao + a];
                                if (with_k) myk[d * nao2 + a * nao + e] += v * D_[b * nao + c];
                            }
                        }
                        (void)n;
                    }
                skip:;
                }
            }
        }
        free(buf);
    }
    size_t tot = (size_t)n_dm * nao2;
    for (size_t x = 0; x < tot; ++x) {
        double sj = 0, sk = 0;
        for (int t = 0; t < nthr; ++t) {
            sj += vj_t[(size_t)t * tot + x];
            sk += vk_t[(size_t)t * tot + x];
        }
        if (vj) vj[x] = sj;
        if (vk) vk[x] = sk;
    }
    if (nquartets) *nquartets = count;
    free(sh); free(q); free(dmc); free(vj_t); free(vk_t);
    return 0;
}

int oracle_jk(const int *atm, const int *bas, int nbas, const double *env,
              const int *ao_loc, const double *dm, int n_dm, double tol,
              int with_j, int with_k, double *vj, double *vk, int nthreads,
              long long *nquartets)
{
    return jk_impl(atm, bas, nbas, env, ao_loc, dm, n_dm, tol, with_j, with_k,
                   vj, vk, nthreads, nquartets, NULL, 0, 0.0);
}

/* The same for the long-range operator erf(omega r)/r (omega > 0); the
 * screening keeps the Coulomb Schwarz bounds, an upper bound of it. */
int oracle_jk_rs(const int *atm, const int *bas, int nbas, const double *env,
                 const int *ao_loc, const double *dm, int n_dm, double tol,
                 int with_j, int with_k, double *vj, double *vk, int nthreads,
                 long long *nquartets, double omega)
{
    return jk_impl(atm, bas, nbas, env, ao_loc, dm, n_dm, tol, with_j, with_k,
                   vj, vk, nthreads, nquartets, NULL, 0, omega);
}

/*
 * The same restricted to the bra shell pairs ij_list (linear index
 * i*(i+1)/2 + j, i >= j; every ket pair kl <= ij of each is visited): a
 * bounded sample of a build, for timing the CPU path on large molecules.
 */
int oracle_jk_sample(const int *atm, const int *bas, int nbas, const double *env,
                     const int *ao_loc, const double *dm, int n_dm, double tol,
                     int with_j, int with_k, double *vj, double *vk, int nthreads,
                     long long *nquartets, const long long *ij_list, long long n_list)
{
    return jk_impl(atm, bas, nbas, env, ao_loc, dm, n_dm, tol, with_j, with_k,
                   vj, vk, nthreads, nquartets, ij_list, n_list, 0.0);
}
