// Device-side data layout and helpers of the B200 J/K engine.
//
// Layout in HBM (all arrays owned by a plan, see jk_api.cu):
//   prim-pair records  double[8] per kept primitive pair
//                      {a_ij, K_ij, Px, Py, Pz, PAx, PAy, PAz}
//                      a_ij = a_i + a_j, K_ij = c_i c_j exp(-a_i a_j/a_ij |AB|^2)
//                      (c with libcint's s/p angular factor folded in),
//                      P the product centre, PA = P - A.
//   shell-pair records PairRec per shell pair, grouped by pair class
//                      (la, lb), la >= lb, each group sorted by q descending.
//   q                  float log(sqrt(max_ab |(ab|ab)|)) per pair record.
//   dm_cond            float log(max |D| over densities, both orientations)
//                      per shell pair, nbas x nbas.
//   densities / J / K  double (n, nao, nao), row-major, Cartesian AO order.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define JK_PI_FAC 34.986836655249725   // 2 pi^(5/2)

struct PairRec {
    int ish, jsh;        // shells; ish carries the higher angular momentum
    int i0, j0;          // first Cartesian AO of each shell
    int prim0, nprim;    // first record and count in the prim-pair table
    float q;             // log Schwarz bound
    float pad;
    double ABx, ABy, ABz;  // A - B, for the i -> j transfer
};

struct ClassArgs {
    const PairRec *bra;      // bra pair class, sorted by q desc
    const PairRec *ket;      // ket pair class, sorted by q desc
    int nbra, nket;
    int same_class;          // bra and ket are the same pair class
    int max_bra_prim;        // largest primitive-pair count of a bra pair
    const double *prim;      // prim-pair records (8 doubles each)
    const double *rys;       // Rys table (double): Chebyshev part + large-x
    const float *rys32;      // Rys table (float)
    const float *dm_cond;    // nbas x nbas
    int nbas;
    float log_tol;
    const float *dm_max;     // device scalar: max of dm_cond
    int nao;
    // K densities: dmK[0..n_ka) then dmKT[0..n_k-n_ka) (the transposes, for
    // non-hermitian builds).  J reads dsJ[0..n_j) = D + D^T.
    const double *dmK;
    const double *dmKT;
    int n_ka, n_k;
    const double *dsJ;
    int n_j;
    double *Kh;              // half-K accumulators (n_k, nao, nao)
    double *Jh;              // half-J accumulators (n_j, nao, nao)
    int *counter;            // work counter for the persistent grid
    unsigned long long *nquartets;  // quartets evaluated (statistics)
    unsigned long long *nprimq;     // primitive quartets evaluated
    float mixed_log_thr;     // mixed precision: quartets whose screened
                             // bound is below this run in FP32 (-inf: off)
    int *error;              // device error flag
};

// ---------------------------------------------------------------------------
// Rys roots and weights from the piecewise Chebyshev table
// (electrolites_b200/codegen/rys_table.py).  Roots are t^2, weights sum to
// F_0(x).  Table layout per order n: [interval][row][coef], rows 0..n-1 the
// roots and n..2n-1 the weights.
// ---------------------------------------------------------------------------
#include "generated/rys_table_dims.inc"

// The large-x nodes (s_k^2) and weights (W_k) follow the Chebyshev part of
// each table: [RYS_LARGEX_OFF + (n-1)*RYS_NMAX + k] roots, then
// [RYS_LARGEX_OFF + RYS_NMAX*RYS_NMAX + ...] weights.
#define RYS_LARGEX_OFF RYS_TABLE_SIZE
#define RYS32_LARGEX_OFF RYS_TABLE32_SIZE
#define RYS_TOTAL (RYS_TABLE_SIZE + 2 * RYS_NMAX * RYS_NMAX)
#define RYS32_TOTAL (RYS_TABLE32_SIZE + 2 * RYS_NMAX * RYS_NMAX)

template <int N>
__device__ __forceinline__ void rys_roots(double x, const double *__restrict__ tab,
                                          double *__restrict__ r,
                                          double *__restrict__ w)
{
    if (x >= RYS_XMAX) {
        double ix = rsqrt(x);
        double inv = ix * ix;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            r[i] = __ldg(tab + RYS_LARGEX_OFF + (N - 1) * RYS_NMAX + i) * inv;
            w[i] = __ldg(tab + RYS_LARGEX_OFF + RYS_NMAX * RYS_NMAX + (N - 1) * RYS_NMAX + i) * ix;
        }
        return;
    }
    int it = (int)(x * RYS_INV_H);
    double s = fma(x - it * RYS_H, 2.0 * RYS_INV_H, -1.0);
    double s2 = s + s;
    const double *c = tab + rys_offset<N>() + it * (2 * N * (RYS_DEGREE + 1));
#pragma unroll
    for (int row = 0; row < 2 * N; ++row) {
        const double2 *cr = reinterpret_cast<const double2 *>(c + row * (RYS_DEGREE + 1));
        // Clenshaw: b_k = c_k + 2 s b_{k+1} - b_{k+2}
        double b1 = 0., b2 = 0.;
#pragma unroll
        for (int k = (RYS_DEGREE + 1) / 2 - 1; k >= 1; --k) {
            double2 cc = __ldg(cr + k);
            double t = fma(s2, b1, cc.y - b2);
            b2 = b1;
            b1 = t;
            t = fma(s2, b1, cc.x - b2);
            b2 = b1;
            b1 = t;
        }
        double2 c0 = __ldg(cr);
        double t = fma(s2, b1, c0.y - b2);
        b2 = b1;
        b1 = t;
        double v = fma(s, b1, c0.x - b2);
        if (row < N) r[row] = v; else w[row - N] = v;
    }
}

// Single-precision variant for the mixed-precision form: a lower-degree
// table, FP32 Clenshaw.  Accuracy ~1e-7 relative.
template <int N>
__device__ __forceinline__ void rys_roots_f32(float x, const float *__restrict__ tab,
                                              float *__restrict__ r,
                                              float *__restrict__ w)
{
    if (x >= (float)RYS_XMAX) {
        float ix = rsqrtf(x);
        float inv = ix * ix;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            r[i] = __ldg(tab + RYS32_LARGEX_OFF + (N - 1) * RYS_NMAX + i) * inv;
            w[i] = __ldg(tab + RYS32_LARGEX_OFF + RYS_NMAX * RYS_NMAX + (N - 1) * RYS_NMAX + i) * ix;
        }
        return;
    }
    int it = (int)(x * (float)RYS_INV_H);
    float s = fmaf(x - it * (float)RYS_H, 2.0f * (float)RYS_INV_H, -1.0f);
    float s2 = s + s;
    const float *c = tab + rys32_offset<N>() + it * (2 * N * (RYS_DEGREE_F32 + 1));
#pragma unroll
    for (int row = 0; row < 2 * N; ++row) {
        const float4 *cr = reinterpret_cast<const float4 *>(c + row * (RYS_DEGREE_F32 + 1));
        float4 hi = __ldg(cr + 1), lo = __ldg(cr);
        float cf[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
        float b1 = 0.f, b2 = 0.f;
#pragma unroll
        for (int k = RYS_DEGREE_F32; k >= 1; --k) {
            float t = fmaf(s2, b1, cf[k] - b2);
            b2 = b1;
            b1 = t;
        }
        float v = fmaf(s, b1, cf[0] - b2);
        if (row < N) r[row] = v; else w[row - N] = v;
    }
}

__device__ __forceinline__ void set_error(int *flag, int code)
{
    if (flag) atomicCAS(flag, 0, code);
}
