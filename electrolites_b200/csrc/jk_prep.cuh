// Preprocessing and post-processing kernels of the J/K engine:
// primitive-pair records, Schwarz bounds, density screening table,
// symmetrised / transposed densities and the final J/K assembly.
#pragma once
#include <cuda_runtime.h>
#include <math.h>
#include "jk_device.cuh"

struct ShellDev {
    double x, y, z;
    int l, nprim;
    int exp_off, coef_off;   // into the device copy of exponents/coefficients
};

#define JK_PRIM_EXP_CUTOFF 60.0   // primitive pairs with a_i a_j/a_ij |AB|^2 > 60 are dropped

// One record per kept primitive pair (JK_PRIM_STRIDE doubles):
// {a_ij, 0.5/a_ij, Kp_ij, P, P - A, 0} with Kp_ij = sqrt(2 pi^5/2) K_ij / a_ij,
// so that the primitive-quartet prefactor 2 pi^5/2 K_ij K_kl /
// (a_ij a_kl sqrt(a_ij + a_kl)) is Kp_ij Kp_kl / sqrt(a_ij + a_kl).
__global__ void prim_pair_fill_kernel(const int4 *__restrict__ rec, long long nrec,
                                      const ShellDev *__restrict__ sh,
                                      const double *__restrict__ basis_data,
                                      double *__restrict__ prim)
{
    long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (r >= nrec) return;
    const int4 q = rec[r];
    const ShellDev A = sh[q.x], B = sh[q.y];
    const double ai = basis_data[A.exp_off + q.z], aj = basis_data[B.exp_off + q.w];
    const double ci = basis_data[A.coef_off + q.z], cj = basis_data[B.coef_off + q.w];
    const double aij = ai + aj;
    const double abx = A.x - B.x, aby = A.y - B.y, abz = A.z - B.z;
    const double rr = abx * abx + aby * aby + abz * abz;
    const double kij = ci * cj * exp(-ai * aj / aij * rr);
    const double t = aj / aij;
    double *o = prim + r * JK_PRIM_STRIDE;
    o[PR_A] = aij;
    o[PR_HIA] = 0.5 / aij;
    o[PR_KP] = JK_SQRT_PI_FAC * kij / aij;
    o[PR_PX] = A.x - t * abx;       // P = A + aj/aij (B - A)
    o[PR_PX + 1] = A.y - t * aby;
    o[PR_PX + 2] = A.z - t * abz;
    o[PR_PAX] = -t * abx;           // P - A
    o[PR_PAX + 1] = -t * aby;
    o[PR_PAX + 2] = -t * abz;
    o[PR_AI] = ai;
}

// FP32 copies of the records (JK_PRIM32_STRIDE floats each) for the mixed
// form's single-precision quartets
__global__ void prim32_fill_kernel(const double *__restrict__ prim, long long nrec,
                                   float *__restrict__ prim32)
{
    const long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (r >= nrec) return;
    const double *in = prim + r * JK_PRIM_STRIDE;
    float *o = prim32 + r * JK_PRIM32_STRIDE;
#pragma unroll
    for (int f = 0; f < JK_PRIM32_STRIDE; ++f) o[f] = f < 9 ? (float)in[f] : 0.f;
}

// The field-major copy of the records (JK_SOA_FIELDS, PairRec::soa): one
// thread per pair of the class lists
__global__ void prim_soa_fill_kernel(const PairRec *__restrict__ pairs, long long npairs,
                                     const double *__restrict__ prim, double *__restrict__ soa)
{
    const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    const PairRec r = pairs[p];
    for (int k = 0; k < r.nprim; ++k) {
        const double *in = prim + (size_t)(r.prim0 + k) * JK_PRIM_STRIDE;
#pragma unroll
        for (int f = 0; f < JK_SOA_FIELDS; ++f)
            soa[r.soa + (size_t)(k * JK_SOA_FIELDS + f) * r.soa_n] = in[f];
    }
}

// ---------------------------------------------------------------------------
// Schwarz bound per shell pair: q = log sqrt(max_ab |(ab|ab)|), with a
// runtime-l Rys evaluation (l <= 3).  One thread per pair; O(npairs) work.
// ---------------------------------------------------------------------------
__device__ inline int ncart_d(int l) { return (l + 1) * (l + 2) / 2; }

__device__ inline void cart_comp_d(int l, int n, int &lx, int &ly, int &lz)
{
    int c = 0;
    for (int x = l; x >= 0; --x)
        for (int y = l - x; y >= 0; --y) {
            if (c == n) { lx = x; ly = y; lz = l - x - y; return; }
            ++c;
        }
    lx = ly = lz = 0;
}

__device__ inline void rys_roots_rt(int n, double x, const double *tab, double *r, double *w)
{
    switch (n) {
    case 1: rys_roots<1>(x, tab, r, w); break;
    case 2: rys_roots<2>(x, tab, r, w); break;
    case 3: rys_roots<3>(x, tab, r, w); break;
    case 4: rys_roots<4>(x, tab, r, w); break;
    case 5: rys_roots<5>(x, tab, r, w); break;
    case 6: rys_roots<6>(x, tab, r, w); break;
    default: rys_roots<7>(x, tab, r, w); break;
    }
}

__global__ void schwarz_kernel(const int4 *__restrict__ pairs, int npairs,
                               const ShellDev *__restrict__ sh,
                               const double *__restrict__ prim,
                               const double *__restrict__ rys, float *__restrict__ q_out)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    const int4 pr = pairs[p];   // ish, jsh, prim0, nprim
    const ShellDev A = sh[pr.x], B = sh[pr.y];
    const int li = A.l, lj = B.l, lij = li + lj;
    const int nroots = lij + 1;
    const int ni = ncart_d(li), nj = ncart_d(lj);
    const double AB[3] = {A.x - B.x, A.y - B.y, A.z - B.z};
    double diag[100];
    for (int n = 0; n < ni * nj; ++n) diag[n] = 0.;
    double G[7][7], Ib[4][4][7], I[3][4][4][4][4];
    double r[7], w[7];
    for (int kp = 0; kp < pr.w; ++kp) {
        const double *K = prim + (size_t)(pr.z + kp) * JK_PRIM_STRIDE;
        const double akl = K[PR_A];
        for (int bp = 0; bp < pr.w; ++bp) {
            const double *P = prim + (size_t)(pr.z + bp) * JK_PRIM_STRIDE;
            const double aij = P[PR_A];
            const double PQ[3] = {P[PR_PX] - K[PR_PX], P[PR_PX + 1] - K[PR_PX + 1],
                                  P[PR_PX + 2] - K[PR_PX + 2]};
            const double s = aij + akl;
            const double rr = PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2];
            const double x = aij * akl / s * rr;
            const double pref = P[PR_KP] * K[PR_KP] / sqrt(s);
            rys_roots_rt(nroots, x, rys, r, w);
            for (int ir = 0; ir < nroots; ++ir) {
                const double u = r[ir];
                const double up = u * akl / s, uq = u * aij / s;
                const double b00 = 0.5 * u / s;
                const double b10 = 0.5 / aij * (1 - up);
                const double b01 = 0.5 / akl * (1 - uq);
                for (int d = 0; d < 3; ++d) {
                    const double c0 = P[PR_PAX + d] - up * PQ[d];
                    const double cp = K[PR_PAX + d] + uq * PQ[d];
                    G[0][0] = d == 2 ? w[ir] * pref : 1.0;
                    for (int e = 0; e < lij; ++e)
                        G[e + 1][0] = c0 * G[e][0] + (e ? e * b10 * G[e - 1][0] : 0.);
                    for (int f = 0; f < lij; ++f)
                        for (int e = 0; e <= lij; ++e)
                            G[e][f + 1] = cp * G[e][f] + (f ? f * b01 * G[e][f - 1] : 0.) +
                                          (e ? e * b00 * G[e - 1][f] : 0.);
                    for (int f = 0; f <= lij; ++f) {
                        double t[7][4];
                        for (int e = 0; e <= lij; ++e) t[e][0] = G[e][f];
                        for (int b = 1; b <= lj; ++b)
                            for (int a = 0; a <= lij - b; ++a)
                                t[a][b] = t[a + 1][b - 1] + AB[d] * t[a][b - 1];
                        for (int a = 0; a <= li; ++a)
                            for (int b = 0; b <= lj; ++b) Ib[a][b][f] = t[a][b];
                    }
                    for (int a = 0; a <= li; ++a)
                        for (int b = 0; b <= lj; ++b) {
                            double t[7][4];
                            for (int f = 0; f <= lij; ++f) t[f][0] = Ib[a][b][f];
                            for (int dd = 1; dd <= lj; ++dd)
                                for (int c = 0; c <= lij - dd; ++c)
                                    t[c][dd] = t[c + 1][dd - 1] + AB[d] * t[c][dd - 1];
                            for (int c = 0; c <= li; ++c)
                                for (int dd = 0; dd <= lj; ++dd) I[d][a][b][c][dd] = t[c][dd];
                        }
                }
                for (int ia = 0; ia < ni; ++ia) {
                    int ax, ay, az;
                    cart_comp_d(li, ia, ax, ay, az);
                    for (int ib = 0; ib < nj; ++ib) {
                        int bx, by, bz;
                        cart_comp_d(lj, ib, bx, by, bz);
                        diag[ia * nj + ib] += I[0][ax][bx][ax][bx] * I[1][ay][by][ay][by] *
                                              I[2][az][bz][az][bz];
                    }
                }
            }
        }
    }
    double m = 0.;
    for (int n = 0; n < ni * nj; ++n) m = fmax(m, fabs(diag[n]));
    q_out[p] = m > 0. ? (float)(0.5 * log(m)) : -INFINITY;
}

// ---------------------------------------------------------------------------
// Density preparation and J/K assembly over every item of a build (one plan
// and its densities per item; a single build is a batch of one).  Each
// launch walks a list of descriptors; a block finds its descriptor by a
// binary search over the descriptors' first block.
// ---------------------------------------------------------------------------

// out[d] = a[d] + f * b[d]^T and outT[d] = b[d]^T for d < nd, n x n
// matrices in 32 x 32 tiles.  A NULL a or b reads as zero; a NULL out or
// outT is not written.  Used with a = b = D for D + D^T (+ D^T) and with the
// half-J/K accumulators for the final J/K.
struct TileOp {
    const double *a;
    const double *b;
    double *out;
    double *outT;
    double f;
    int n, nd;
    int nt;             // tiles per side, ceil(n / 32)
    long long tile0;    // first block of this op in the launch
};

// Two densities interleaved element by element, out[i] = (a[i], b[i]): the
// register digest of a build with two or more K densities reads both
// densities of a pair with one 16-byte load.
struct PairOp {
    const double *a;
    const double *b;
    double2 *out;
    long long n;        // elements of one density (nao^2)
    long long blk0;     // first block of this op in the launch
};

#define JK_PAIR_THREADS 256

__global__ void pair_dens_kernel(const PairOp *__restrict__ ops, int nops)
{
    const long long blk = blockIdx.x;
    int lo = 0, hi = nops - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (ops[mid].blk0 <= blk) lo = mid; else hi = mid - 1;
    }
    const PairOp o = ops[lo];
    const long long i = (blk - o.blk0) * JK_PAIR_THREADS + threadIdx.x;
    if (i < o.n) o.out[i] = make_double2(o.a[i], o.b[i]);
}

__global__ void tile_op_kernel(const TileOp *__restrict__ ops, int nops)
{
    __shared__ double tile[32][33];
    const long long t = blockIdx.x;
    int lo = 0, hi = nops - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (ops[mid].tile0 <= t) lo = mid; else hi = mid - 1;
    }
    const TileOp o = ops[lo];
    long long r = t - o.tile0;
    const long long per = (long long)o.nt * o.nt;
    const int d = (int)(r / per);
    r -= d * per;
    const int n = o.n;
    const size_t n2 = (size_t)n * n;
    const int bx = (int)(r / o.nt) * 32, by = (int)(r % o.nt) * 32;
    const double *y = o.b ? o.b + d * n2 : nullptr;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int rr = bx + k, c = by + threadIdx.x;     // b[rr][c], coalesced
        tile[k][threadIdx.x] = (y && rr < n && c < n) ? y[(size_t)rr * n + c] : 0.;
    }
    __syncthreads();
    const double *x = o.a ? o.a + d * n2 : nullptr;
    double *out = o.out ? o.out + d * n2 : nullptr;
    double *outT = o.outT ? o.outT + d * n2 : nullptr;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int rr = by + k, c = bx + threadIdx.x;     // (b^T)[rr][c] = tile[tx][k]
        if (rr < n && c < n) {
            const double bt = tile[threadIdx.x][k];
            const size_t idx = (size_t)rr * n + c;
            if (out) out[idx] = (x ? x[idx] : 0.) + o.f * bt;
            if (outT) outT[idx] = bt;
        }
    }
}

// Density screening table of one item:
// dm_cond[ish][jsh] = log max |D[d][a][b]|, |D[d][b][a]| over its densities
// and the shells' AOs (symmetric by construction), its maximum dm_max, and
// the range check against the pairs the plan dropped.
struct CondItem {
    const double *dm;
    const int *sh_ao;
    const int *sh_nf;
    float *dmc;
    float *dm_max;
    int n_dm, nao, nbas;
    int nt;             // 16 x 16 shell tiles per side
    long long blk0;     // first block of this item in the launch
    float q_drop;       // largest Schwarz bound of a pair the plan dropped
    float q_max;        // largest Schwarz bound of the plan
    float log_tol;
    int pad;
};

__global__ void dm_cond_kernel(const CondItem *__restrict__ items, int nitems)
{
    const long long t = blockIdx.x;
    int lo = 0, hi = nitems - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (items[mid].blk0 <= t) lo = mid; else hi = mid - 1;
    }
    const CondItem it = items[lo];
    const int r = (int)(t - it.blk0);
    const int i = (r / it.nt) * 16 + threadIdx.y;
    const int j = (r % it.nt) * 16 + threadIdx.x;
    const int nbas = it.nbas, nao = it.nao;
    if (i >= nbas || j >= nbas) return;
    const int a0 = __ldg(it.sh_ao + i), na = __ldg(it.sh_nf + i);
    const int b0 = __ldg(it.sh_ao + j), nb = __ldg(it.sh_nf + j);
    const size_t nao2 = (size_t)nao * nao;
    double m = 0.;
    for (int d = 0; d < it.n_dm; ++d) {
        const double *D = it.dm + d * nao2;
        for (int a = 0; a < na; ++a)
            for (int b = 0; b < nb; ++b) {
                m = fmax(m, fabs(D[(size_t)(a0 + a) * nao + b0 + b]));
                m = fmax(m, fabs(D[(size_t)(b0 + b) * nao + a0 + a]));
            }
    }
    it.dmc[(size_t)i * nbas + j] = m > 0. ? (float)log(m) : -INFINITY;
}

// one block per item: dm_max, and err = {JK_ERR_RANGE, item} if a pair the
// plan dropped could pass the screening with this density
// (q_drop + q_max + dm_max > log_tol)
__global__ void dm_max_kernel(const CondItem *__restrict__ items, int *__restrict__ err)
{
    __shared__ float s[256];
    const CondItem it = items[blockIdx.x];
    const long long n = (long long)it.nbas * it.nbas;
    float m = -INFINITY;
    for (long long k = threadIdx.x; k < n; k += blockDim.x) m = fmaxf(m, it.dmc[k]);
    s[threadIdx.x] = m;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) s[threadIdx.x] = fmaxf(s[threadIdx.x], s[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        *it.dm_max = s[0];
        if (it.q_drop + it.q_max + s[0] > it.log_tol && atomicCAS(err, 0, 5) == 0)
            err[1] = blockIdx.x;
    }
}

// Rows of the task decomposition: one per (view v, bra pair b, ket sub-list
// s), r = row0(v) + b * nsub(v) + s.  row_ncand[r] = kets of sub-list s
// (ordered by Schwarz bin) in the bins that can pass the Schwarz test with
// the plan's largest density element, limited to ket index <= b within a
// diagonal class.
__global__ void task_rows_kernel(const ClassArgs a, int *__restrict__ row_ncand)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= a.nrows) return;
    int lo = 0, hi = a.nviews - 1;
    while (lo < hi) {                    // last view with row0 <= r
        const int mid = (lo + hi + 1) >> 1;
        if (a.view_row0[mid] <= r) lo = mid; else hi = mid - 1;
    }
    const PlanView &V = a.views[lo];
    const int rl = r - V.row0;
    const int b = rl / V.nsub, s = rl - (rl / V.nsub) * V.nsub;
    // candidates: the kets of every Schwarz bin from the top down to the bin
    // of the cut (pairs are sorted by bin within a sub-list; the cut's bin is
    // screened quartet by quartet)
    const float cut = jk_qbin(V.log_tol - V.bra[b].q - *V.dm_max);
    lo = V.sub[s].x;
    hi = V.sub[s].y;
    if (V.same_class && hi > b + 1) hi = b + 1;
    const int first = lo;
    if (lo > hi) hi = lo;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (jk_qbin(V.ket[mid].q) >= cut) lo = mid + 1; else hi = mid;
    }
    row_ncand[r] = lo - first;
}

// Task size from the class's total candidate count (cand_prefix[rows-1]):
// about `target` tasks, clamped to [lo, hi] kets and rounded to a warp; then
// the chunk count of every row.  Grouped classes (a.grouped) count the
// chunks of a bra pair's candidates over all its ket sub-lists on the bra's
// first row (sub-list 0) and none on its other rows.
__global__ void task_chunks_kernel(const ClassArgs a, const int *__restrict__ ncand,
                                   const int *__restrict__ cand_prefix, int rows, int target,
                                   int lo, int hi, int *__restrict__ chunk_out,
                                   int *__restrict__ chunks)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    const long long total = rows > 0 ? cand_prefix[rows - 1] : 0;
    long long c = (total + target - 1) / target;
    c = (c + 31) / 32 * 32;
    if (c < lo) c = lo;
    if (c > hi) c = hi;
    if (r == 0) *chunk_out = (int)c;
    if (r >= rows) return;
    if (!a.grouped) {
        chunks[r] = (int)((ncand[r] + c - 1) / c);
        return;
    }
    int vlo = 0, vhi = a.nviews - 1;
    while (vlo < vhi) {                  // last view with row0 <= r
        const int mid = (vlo + vhi + 1) >> 1;
        if (a.view_row0[mid] <= r) vlo = mid; else vhi = mid - 1;
    }
    const PlanView &V = a.views[vlo];
    const int s = (r - V.row0) % V.nsub;
    if (s != 0) {
        chunks[r] = 0;
        return;
    }
    const long long g = cand_prefix[r + V.nsub - 1] - (r > 0 ? cand_prefix[r - 1] : 0);
    chunks[r] = (int)((g + c - 1) / c);
}
