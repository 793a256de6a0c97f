// Device-side data layout and helpers of the B200 J/K engine.
//
// Layout in HBM (all arrays owned by a plan, see jk_api.cu):
//   prim-pair records  double[JK_PRIM_STRIDE] per kept primitive pair
//                      {a_ij, 1/(2 a_ij), Kp_ij, Px, Py, Pz, PAx, PAy, PAz, 0}
//                      a_ij = a_i + a_j, K_ij = c_i c_j exp(-a_i a_j/a_ij |AB|^2)
//                      (c with libcint's s/p angular factor folded in),
//                      Kp_ij = sqrt(2 pi^(5/2)) K_ij / a_ij,
//                      P the product centre, PA = P - A.
//   shell-pair records PairRec per shell pair, grouped by pair class
//                      (la, lb), la >= lb, each group in sub-lists of equal
//                      primitive count ordered by Schwarz bin (JK_QBIN_W).
//   q                  float log(sqrt(max_ab |(ab|ab)|)) per pair record.
//   dm_cond            float log(max |D| over densities, both orientations)
//                      per shell pair, nbas x nbas.
//   x-space blocks     J engine: per shell pair P of class (la, lb), n_j x
//                      NX doubles, NX = sum_{L=la}^{la+lb} ncart(L) (the
//                      source levels of the pair's transfer H^P):
//                      D~_P = H^P^T (D+D^T)_P and the x-space J of P.
//   densities / J / K  double (n, nao, nao), row-major, Cartesian AO order.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#define JK_SQRT_PI_FAC 5.914967172795612    // sqrt(2 pi^(5/2))

// primitive-pair record: JK_PRIM_STRIDE doubles, fields at these offsets
#define JK_PRIM_STRIDE 10
#define PR_A 0      // a_ij
#define PR_HIA 1    // 0.5 / a_ij
#define PR_KP 2     // sqrt(2 pi^5/2) K_ij / a_ij
#define PR_PX 3     // P (3)
#define PR_PAX 6    // P - A (3)
#define PR_AI 9     // a_i, the exponent of the first shell's primitive (gradients)
// FP32 copy of the records for the mixed form's single-precision quartets:
// the same fields as floats, 12 per record (16-byte aligned)
#define JK_PRIM32_STRIDE 12

// Order of the pairs within a sub-list: by the decade of their Schwarz
// bound (q / JK_QBIN_W, JK_QBIN_W = ln 10, descending), then by first and
// second shell.  The bins keep the candidates of a bra pair a prefix of the
// sub-list (every pair of a bin above the cut passes the Schwarz test, the
// cut's own bin is screened per quartet); within a bin, pairs that share
// their first shell k are adjacent, so the K_h[i,k] and K_h[j,k] terms of a
// run of kets accumulate in registers and the density rows D[i,k], D[j,k]
// of neighbouring lanes coincide.
#define JK_QBIN_W 2.302585092994046f
__host__ __device__ __forceinline__ float jk_qbin(float q) { return floorf(q / JK_QBIN_W); }

// McMurchie-Davidson J (jk_mdj.cuh): densities of a build it serves (more:
// the Rys J engine) and the largest l_i + l_j + l_k + l_l of its classes
#define JK_MD_DENS 2
#define JK_MD_LMAX 6

// Cartesian components: count, powers and index of a level (PySCF order)
__host__ __device__ constexpr int g_ncart(int l) { return (l + 1) * (l + 2) / 2; }

// component d (0 x, 1 y, 2 z) of Cartesian function n of level L <= 7
// (PySCF order: lx descending, then ly descending).  Closed form, no loop,
// so that with constant arguments (unrolled loops) every use folds to a
// constant and the arrays it indexes stay in registers.  k = L - lx is the
// group of n (the groups before it hold k (k + 1) / 2 functions); within
// it, lz = n - k (k + 1) / 2.
__host__ __device__ constexpr int g_comp(int L, int n, int d)
{
    const int k = n >= 28 ? 7 : n >= 21 ? 6 : n >= 15 ? 5 : n >= 10 ? 4 : n >= 6 ? 3
                : n >= 3 ? 2 : n >= 1 ? 1 : 0;
    const int lz = n - k * (k + 1) / 2;
    return d == 0 ? L - k : (d == 1 ? k - lz : lz);
}

// index of (lx, ly, lz) within its level
__host__ __device__ constexpr int g_idx(int lx, int ly, int lz)
{
    return (ly + lz) * (ly + lz + 1) / 2 + lz;
}

struct PairRec {
    int ish, jsh;        // shells; ish carries the higher angular momentum
    int i0, j0;          // first Cartesian AO of each shell
    int prim0, nprim;    // first record and count in the prim-pair table
    float q;             // log Schwarz bound
    int xoff;            // first element of this pair's x-space block (J engine)
    int soa, soa_n;      // field-major copy: field f of primitive pair k at
                         // prim_soa[soa + (k * JK_SOA_FIELDS + f) * soa_n]
    double ABx, ABy, ABz;  // A - B, for the i -> j transfer
};

// Field-major copy of the primitive-pair records in ket order (the register
// form's ket loop): per sub-list of n pairs of P primitive pairs each, a
// block of P * JK_SOA_FIELDS rows of n doubles, row (k, f) holding field f
// (PR_* order) of primitive pair k of every pair of the sub-list.  Lanes that
// evaluate neighbouring kets of a sub-list read neighbouring doubles.
#define JK_SOA_FIELDS 9

// One plan (molecule) as one class launch sees it.  A launch covers a list
// of views -- one plan for an ordinary build, hundreds in a batched build --
// and every task names the view it belongs to.
struct PlanView {
    const PairRec *bra;      // bra pair class of this plan (sub-lists, binned)
    const PairRec *ket;      // ket pair class of this plan
    const int2 *sub;         // ket sub-lists [begin, end) within the ket class
    const double *prim;      // prim-pair records of this plan
    const double *prim_soa;  // their field-major copy in ket order
    const float *prim32;     // their FP32 copies
    const float *dm_cond;    // nbas x nbas
    const float *dm_max;     // device scalar: max of dm_cond
    // K densities: dmK[0..n_ka) then dmKT[0..n_k-n_ka) (the transposes, for
    // non-hermitian builds).  J reads dsJ[0..n_j) = D + D^T.
    const double *dmK;
    const double *dmKT;
    // the K densities interleaved in pairs (2p, 2p+1), p < n_k / 2, for the
    // register digest (null: every density read on its own)
    const double2 *dmK2;
    const double *dsJ;
    double *Kh;              // half-K accumulators (n_k, nao, nao)
    double *Jh;              // half-J accumulators (n_j, nao, nao)
    int nbra, nket, nsub, same_class;
    int nbas, nao, n_ka, n_k;
    int n_j;
    float log_tol;
    float mixed_log_thr;     // mixed precision: quartets whose screened
                             // bound is below this run in FP32 (-inf: off)
    int row0;                // first task row of this view in the launch
};

struct ClassArgs {
    const PlanView *views;   // every view of the class (global copy)
    const int *view_row0;    // first task row of each view (binary search)
    int nviews;
    int nrows;
    // the part of the class this launch covers: views [view_begin,
    // view_begin + nvl), task rows [row_begin, row_end)
    int view_begin, nvl, row_begin, row_end;
    int max_bra_prim;        // largest primitive-pair count of a bra pair
    int mixed;               // 1: the build has FP32 quartets (mixed form)
    int mixed_tab;           // 1: the FP32 Rys table is in shared memory (set at launch)
    int shard_rank, shard_size;   // this GPU takes tasks t = rank mod size
    // 1: a task is a range of the concatenated candidate kets of all ket
    // sub-lists of one bra pair (its chunks are counted on the bra's first
    // row), so a warp's queue runs on across sub-lists; 0: one sub-list's
    int grouped;
    // the operator: sum over nterm (1 or 2) terms of op_coef[t] times the
    // Coulomb operator (op_inv_om2[t] = 0) or the long-range erf(omega r)/r
    // (op_inv_om2[t] = 1/omega^2); quartets are screened by the Coulomb bound
    int nterm;
    double op_coef[2];
    double op_inv_om2[2];
    // J engine (single-plan builds): 0 off; 1 = J from each quartet's
    // (e0|f0) block contracted with the pairs' x-space densities (K, if any,
    // from the transfers); 2 = the same in a J-only build.  Pair P's block
    // of n_j x NX(P) doubles starts at P.xoff * n_j in jx_dens (densities)
    // and jx_acc (J)
    int jx;
    const double *jx_dens;
    double *jx_acc;
    // nuclear gradient (grad != null): dE/dR per atom, natm x 3, for
    // W = fac [grad_wj Dt_ab Dt_cd - grad_wk sum_s (D_ac D_bd + D_ad D_bc)];
    // sh_atom: the atom of every shell of the plan
    double *grad;
    const int *sh_atom;
    double grad_wj, grad_wk;
    int natm;            // atoms of the plan (forces of up to JK_GRAD_SMEM_ATOMS
                         // atoms are summed per block in shared memory)
    const double *rys;       // Rys table (double): polynomial part + large-x
    const float *rys32;      // Rys table (float)
    int *counter;            // task counter of this launch
    const int *chunk;        // kets per task (device scalar, set per launch)
    const int *row_ncand;    // candidate kets per row
    const int *row_prefix;   // inclusive prefix sum of chunks per row
    unsigned long long *nquartets;  // quartets evaluated (statistics)
    unsigned long long *nprimq;     // primitive quartets evaluated
    unsigned long long *nquartets32;  // quartets evaluated in FP32
};

// Views per launch of a batched class: the launch carries its views in its
// kernel parameters (__grid_constant__, read through the constant cache, so
// a view field costs no register while it is not in use).  Kernel
// parameters may hold 32764 bytes.
#define JK_VTAB 192

template <int NV>
struct LaunchParams {
    ClassArgs a;
    PlanView v[NV];
};
static_assert(sizeof(LaunchParams<JK_VTAB>) <= 32000, "kernel parameters hold at most 32764 bytes");

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

// Interval index and local variable s in [-1, 1] of x < RYS_XMAX.  The
// segment is picked by comparison and floor((x - x0)/h) by adding 1.5*2^52,
// which leaves the rounded integer in the low mantissa bits: no
// double-to-int conversion, which would run on the XU pipe that the rsqrt
// of every primitive quartet already occupies.
__device__ __forceinline__ void rys_locate(double x, int &it, double &s)
{
    const bool g1 = x >= RYS_SEG1, g2 = x >= RYS_SEG2;
    const double x0 = g2 ? RYS_SEG2 : (g1 ? RYS_SEG1 : 0.0);
    const double ih = g2 ? RYS_IH2 : (g1 ? RYS_IH1 : RYS_IH0);
    const int it0 = g2 ? RYS_IT2 : (g1 ? RYS_IT1 : 0);
    const double v = (x - x0) * ih;
    const double y = (v - 0.5) + 6755399441055744.0;     // 1.5 * 2^52
    const double fk = y - 6755399441055744.0;
    it = it0 + __double2loint(y);
    s = 2.0 * (v - fk) - 1.0;
}

__device__ __forceinline__ void rys_locate_f32(float x, int &it, float &s)
{
    const bool g1 = x >= (float)RYS_SEG1, g2 = x >= (float)RYS_SEG2;
    const float x0 = g2 ? (float)RYS_SEG2 : (g1 ? (float)RYS_SEG1 : 0.0f);
    const float ih = g2 ? (float)RYS_IH2 : (g1 ? (float)RYS_IH1 : (float)RYS_IH0);
    const int it0 = g2 ? RYS_IT2 : (g1 ? RYS_IT1 : 0);
    const float v = (x - x0) * ih;
    const float y = (v - 0.5f) + 12582912.0f;             // 1.5 * 2^23
    const float fk = y - 12582912.0f;
    it = it0 + (__float_as_int(y) & 0x3fffff);
    s = 2.0f * (v - fk) - 1.0f;
}

// One table row, sum_k c_k s^k with k < 8, by Estrin's scheme (depth 3).
__device__ __forceinline__ double rys_poly8(const double2 *__restrict__ cr, double s,
                                            double s2, double s4)
{
    const double2 c01 = __ldg(cr), c23 = __ldg(cr + 1), c45 = __ldg(cr + 2);
    const double2 c67 = __ldg(cr + 3);
    const double p0 = fma(c01.y, s, c01.x), p1 = fma(c23.y, s, c23.x);
    const double p2 = fma(c45.y, s, c45.x), p3 = fma(c67.y, s, c67.x);
    return fma(fma(p3, s2, p2), s4, fma(p1, s2, p0));
}

template <int N>
__device__ __forceinline__ void rys_roots(double x, const double *__restrict__ tab,
                                          double *__restrict__ r,
                                          double *__restrict__ w)
{
    static_assert(RYS_DEGREE == 7, "rys_poly8 evaluates degree 7");
    if (x >= rys_xmax<N>()) {
        double ix = rsqrt(x);
        double inv = ix * ix;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            r[i] = __ldg(tab + RYS_LARGEX_OFF + (N - 1) * RYS_NMAX + i) * inv;
            w[i] = __ldg(tab + RYS_LARGEX_OFF + RYS_NMAX * RYS_NMAX + (N - 1) * RYS_NMAX + i) * ix;
        }
        return;
    }
    int it;
    double s;
    rys_locate(x, it, s);
    const double s2 = s * s, s4 = s2 * s2;
    const double2 *c = reinterpret_cast<const double2 *>(
        tab + rys_offset<N>() + it * (2 * N * (RYS_DEGREE + 1)));
#pragma unroll
    for (int row = 0; row < 2 * N; ++row) {
        const double v = rys_poly8(c + row * (RYS_DEGREE + 1) / 2, s, s2, s4);
        if (row < N) r[row] = v; else w[row - N] = v;
    }
}
