// Nuclear gradient of the two-electron energy, one class per launch.
//
// For symmetric densities D_s (s < n_dm), Dt = sum_s D_s, held fixed in the
// AO basis while the atoms move,
//   E = j/2 Tr[Dt J[Dt]] - k c sum_s Tr[D_s K[D_s]]   (c = 1/4 for one density,
//                                                       1/2 for two)
// -- the energy whose per-atom derivative GPU4PySCF's _jk_energy_per_atom
// returns and the reference replaces (electrolites/fastejk.py:276-356, its
// factors at :308-316).  Over the distinct permutations of a unique shell
// quartet with degeneracy factor sf, E collects sum_abcd W_abcd (ab|cd),
//   W = sf [4 j Dt_ab Dt_cd - 4 k c sum_s (D_s,ac D_s,bd + D_s,ad D_s,bc)],
// and d/dA_x of a Cartesian Gaussian on A is 2 alpha g_{a+1x} - a_x g_{a-1x},
// so dE/dA = sum W (d(ab|cd)/dA) needs the quartet's integrals with shell i
// raised (weighted by 2 alpha_i per primitive) and lowered by one; likewise
// j and k; the centre of l follows from translational invariance,
// dD = -(dA + dB + dC).
//
// Work decomposition: the register form's (tasks of a bra pair against a
// range of kets, one quartet per lane, claimed per warp).  Forces are summed
// per block in shared memory (molecules of up to JK_GRAD_SMEM_ATOMS atoms)
// and added to the output once per block and atom component: every quartet
// adds to the same natm x 3 numbers, so global atomics per quartet would all
// contend for a few hundred addresses.  Two forms, chosen per class by
// measurement in the code generator (G_SMALL):
//   per lane: per quartet, primitive quartet and Rys root, the generated
//   grad_root adds the root's 2D-integral products to four (e|f)-space
//   blocks in registers: U (unweighted), RA, RB, RC (weighted by 2 alpha of
//   the primitive of shell i, j, k); after the primitive sums the generated
//   transfers of the shifted shells give each derivative block, which is
//   contracted with W on the fly.  Classes with many block products
//   (G_SPLIT) run one primitive pass per block so that one block is live at
//   a time (four blocks spilled to local memory).  The bra atoms' forces add
//   up in registers over a task; the ket atoms' go to the block's sums per
//   quartet;
//   per warp (the larger classes): see grad_team_quartet below.
#pragma once

// atoms whose forces a block sums in shared memory (24 KB) before adding
// them to the output; larger molecules add every quartet's forces there
#define JK_GRAD_SMEM_ATOMS 1024


// derivative block X (nab x NKL, a at level la, rows (a * NB + b)) of a
// shifted shell, contracted with W over the class's (a, b, c, d): for the
// raised shell (sign +1) X[a + 1x], for the lowered one (-1) a_x X[a - 1x].
// POS 0: shell i (a shifted), 1: shell j (b shifted); the ket positions
// are handled by grad_ket_contract.
template <class C, int POS, int LSH, int SIGN>
__device__ __forceinline__ void grad_bra_contract(const double *X, const double *Wt, double g[3])
{
        constexpr int NI = C::NI, NJ = C::NJ, NKL = C::NK * C::NL;
    constexpr int LA = POS == 0 ? C::LI : C::LJ;      // the unshifted level
    constexpr int NA = g_ncart(LA), NSH = g_ncart(LSH);
#pragma unroll
    for (int a = 0; a < NA; ++a) {
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            int c[3] = {g_comp(LA, a, 0), g_comp(LA, a, 1), g_comp(LA, a, 2)};
            const int nx = c[x];
            if (SIGN < 0 && nx == 0) continue;
            c[x] += SIGN;
            const int as = g_idx(c[0], c[1], c[2]);
            const double f = SIGN > 0 ? 1.0 : -(double)nx;
            double s = 0.;
#pragma unroll
            for (int o = 0; o < (POS == 0 ? NJ : NI); ++o) {
                // POS 0: W row (a, b = o), X row (as, o); POS 1: W (i = o, a), X (o, as)
                const int wrow = POS == 0 ? a * NJ + o : o * NJ + a;
                const int xrow = POS == 0 ? as * NJ + o : o * NSH + as;
#pragma unroll
                for (int kl = 0; kl < NKL; ++kl) s = fma(Wt[wrow * NKL + kl], X[xrow * NKL + kl], s);
            }
            g[x] = fma(f, s, g[x]);
        }
    }
}

// the same for shell k (c shifted): X[(ij) * (NSH * NL) + cs * NL + d]
template <class C, int LSH, int SIGN>
__device__ __forceinline__ void grad_ket_contract(const double *X, const double *Wt, double g[3])
{
        constexpr int NIJ = C::NI * C::NJ, NK = C::NK, NL = C::NL;
    constexpr int LC = C::LK, NSH = g_ncart(LSH);
#pragma unroll
    for (int c = 0; c < NK; ++c) {
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            int q[3] = {g_comp(LC, c, 0), g_comp(LC, c, 1), g_comp(LC, c, 2)};
            const int nx = q[x];
            if (SIGN < 0 && nx == 0) continue;
            q[x] += SIGN;
            const int cs = g_idx(q[0], q[1], q[2]);
            const double f = SIGN > 0 ? 1.0 : -(double)nx;
            double s = 0.;
#pragma unroll
            for (int ij = 0; ij < NIJ; ++ij)
#pragma unroll
                for (int d = 0; d < NL; ++d)
                    s = fma(Wt[(ij * NK + c) * NL + d], X[(ij * NSH + cs) * NL + d], s);
            g[x] = fma(f, s, g[x]);
        }
    }
}

// bra-shifted block: R (f-major, NE_R e components from the transfer's first
// level, nf = the class's f components) -> X[(a b) * NKL + kl] via the
// shifted bra transfer and the class's ket transfer
template <class C, int NAB, class HB>
__device__ __forceinline__ void grad_bra_block(const double *R, int ne, HB hb,
                                               const PairRec &br, const PairRec &kt, double *X)
{
        constexpr int NF = C::NF, NKL = C::NK * C::NL;
    double tb[NF * NAB];
#pragma unroll
    for (int f = 0; f < NF; ++f) hb(R + f * ne, tb + f * NAB, br.ABx, br.ABy, br.ABz);
#pragma unroll
    for (int ab = 0; ab < NAB; ++ab) {
        double row[NF];
#pragma unroll
        for (int f = 0; f < NF; ++f) row[f] = tb[f * NAB + ab];
        C::template hrr_ket<double>(row, X + ab * NKL, kt.ABx, kt.ABy, kt.ABz);
    }
}

// The primitive loop of one quartet: per primitive quartet and Rys root the
// generated root routine adds to the blocks.  R = -1: all four blocks at once
// (grad_root); R = 0..3: U, RA, RB or RC alone (the split classes'
// grad_root_U .. grad_root_RC; the other pointers are unused).
template <class C, int R>
__device__ __forceinline__ void grad_accum(const ClassArgs &A, const PlanView &V,
                                           const PairRec &br, const PairRec &kt,
                                           const double *__restrict__ sbra, double *U, double *RA,
                                           double *RB, double *RC)
{
    constexpr int NR = C::G_NROOTS;
    const double io2 = A.op_inv_om2[0];
    const double *cheb = A.rys + rys_offset<NR>();
    for (int kp = 0; kp < kt.nprim; ++kp) {
        const double *kr = V.prim + (size_t)(kt.prim0 + kp) * JK_PRIM_STRIDE;
        const double akl = __ldg(kr + PR_A), hiq = __ldg(kr + PR_HIA), kq = __ldg(kr + PR_KP);
        const double Qx = __ldg(kr + PR_PX), Qy = __ldg(kr + PR_PX + 1), Qz = __ldg(kr + PR_PX + 2);
        const double QCx = __ldg(kr + PR_PAX), QCy = __ldg(kr + PR_PAX + 1), QCz = __ldg(kr + PR_PAX + 2);
        const double wC = 2.0 * __ldg(kr + PR_AI);
        for (int bp = 0; bp < br.nprim; ++bp) {
            const double *s = sbra + bp * JK_PRIM_STRIDE;
            const double aij = s[PR_A], hip = s[PR_HIA];
            const double wA = 2.0 * s[PR_AI], wB = 2.0 * (aij - s[PR_AI]);
            const double PQx = s[PR_PX] - Qx, PQy = s[PR_PX + 1] - Qy, PQz = s[PR_PX + 2] - Qz;
            const double rs = rsqrt(fma(aij * akl, io2, aij + akl));
            const double is = rs * rs;
            const double x = aij * akl * is * fma(PQx, PQx, fma(PQy, PQy, PQz * PQz));
            const double pref = s[PR_KP] * kq * rs;
            double r[NR], w[NR];
            rys_eval<NR, false>(x, cheb, A.rys, r, w);
            const double PAx = s[PR_PAX], PAy = s[PR_PAX + 1], PAz = s[PR_PAX + 2];
#pragma unroll
            for (int n = 0; n < NR; ++n) {
                const double uis = r[n] * is;
                const double up = uis * akl, uq = uis * aij;
                const double c0x = fma(-up, PQx, PAx), c0y = fma(-up, PQy, PAy);
                const double c0z = fma(-up, PQz, PAz), cpx = fma(uq, PQx, QCx);
                const double cpy = fma(uq, PQy, QCy), cpz = fma(uq, PQz, QCz);
                const double b10 = fma(-hip, up, hip), b01 = fma(-hiq, uq, hiq);
                const double wz = w[n] * pref, b00 = 0.5 * uis;
                if constexpr (R < 0)
                    C::template grad_root<double>(c0x, c0y, c0z, cpx, cpy, cpz, b00, b10, b01, wz,
                                                  wA, wB, wC, U, RA, RB, RC);
                else if constexpr (R == 0)
                    C::template grad_root_U<double>(c0x, c0y, c0z, cpx, cpy, cpz, b00, b10, b01, wz,
                                                    1.0, U);
                else if constexpr (R == 1)
                    C::template grad_root_RA<double>(c0x, c0y, c0z, cpx, cpy, cpz, b00, b10, b01, wz,
                                                     wA, RA);
                else if constexpr (R == 2)
                    C::template grad_root_RB<double>(c0x, c0y, c0z, cpx, cpy, cpz, b00, b10, b01, wz,
                                                     wB, RB);
                else
                    C::template grad_root_RC<double>(c0x, c0y, c0z, cpx, cpy, cpz, b00, b10, b01, wz,
                                                     wC, RC);
            }
        }
    }
}

// W = fac [wj Dt_ab Dt_cd - wk sum_s (D_ac D_bd + D_ad D_bc)], Dt = (D + D^T)/2 summed
template <class C>
__device__ __forceinline__ void grad_w(const ClassArgs &A, const PlanView &V, const PairRec &br,
                                       const PairRec &kt, double fac, double *Wt)
{
    constexpr int NI = C::NI, NJ = C::NJ, NK = C::NK, NL = C::NL;
    constexpr int NIJ = NI * NJ, NKL = NK * NL;
    const size_t nao = V.nao, nao2 = nao * nao;
    const int i0 = br.i0, j0 = br.j0, k0 = kt.i0, l0 = kt.j0;
    {
        double dab[NIJ], dcd[NKL];
#pragma unroll
        for (int a = 0; a < NI; ++a)
#pragma unroll
            for (int b = 0; b < NJ; ++b) dab[a * NJ + b] = 0.;
#pragma unroll
        for (int c = 0; c < NKL; ++c) dcd[c] = 0.;
        for (int d = 0; d < V.n_j; ++d) {
            const double *ds = V.dsJ + d * nao2;
#pragma unroll
            for (int a = 0; a < NI; ++a)
#pragma unroll
                for (int b = 0; b < NJ; ++b) dab[a * NJ + b] += 0.5 * __ldg(ds + (i0 + a) * nao + j0 + b);
#pragma unroll
            for (int c = 0; c < NK; ++c)
#pragma unroll
                for (int e = 0; e < NL; ++e) dcd[c * NL + e] += 0.5 * __ldg(ds + (k0 + c) * nao + l0 + e);
        }
        const double wj = A.grad_wj * fac;
#pragma unroll
        for (int ab = 0; ab < NIJ; ++ab)
#pragma unroll
            for (int cd = 0; cd < NKL; ++cd) Wt[ab * NKL + cd] = wj * dab[ab] * dcd[cd];
    }
    const double wk = A.grad_wk * fac;
    for (int d = 0; d < V.n_k; ++d) {
        const double *D = V.dmK + d * nao2;
        double dac[NI * NK], dbd[NJ * NL], dad[NI * NL], dbc[NJ * NK];
#pragma unroll
        for (int a = 0; a < NI; ++a) {
#pragma unroll
            for (int c = 0; c < NK; ++c) dac[a * NK + c] = __ldg(D + (i0 + a) * nao + k0 + c);
#pragma unroll
            for (int e = 0; e < NL; ++e) dad[a * NL + e] = __ldg(D + (i0 + a) * nao + l0 + e);
        }
#pragma unroll
        for (int b = 0; b < NJ; ++b) {
#pragma unroll
            for (int e = 0; e < NL; ++e) dbd[b * NL + e] = __ldg(D + (j0 + b) * nao + l0 + e);
#pragma unroll
            for (int c = 0; c < NK; ++c) dbc[b * NK + c] = __ldg(D + (j0 + b) * nao + k0 + c);
        }
#pragma unroll
        for (int a = 0; a < NI; ++a)
#pragma unroll
            for (int b = 0; b < NJ; ++b)
#pragma unroll
                for (int c = 0; c < NK; ++c)
#pragma unroll
                    for (int e = 0; e < NL; ++e)
                        Wt[((a * NJ + b) * NK + c) * NL + e] -=
                            wk * fma(dac[a * NK + c], dbd[b * NL + e], dad[a * NL + e] * dbc[b * NK + c]);
    }
}

// the derivative contributions of each block, contracted with W
// U: shells i, j and k lowered
template <class C>
__device__ __forceinline__ void grad_from_u(const double *U, const double *Wt, const PairRec &br,
                                            const PairRec &kt, double gA[3], double gB[3],
                                            double gC[3])
{
    constexpr int LI = C::LI, LJ = C::LJ, LK = C::LK, LL = C::LL;
    constexpr int NI = C::NI, NJ = C::NJ, NL = C::NL, NIJ = NI * NJ, NKL = C::NK * NL;
    if constexpr (LI > 0) {
        constexpr int NAB = g_ncart(LI - 1) * NJ;
        double X[NAB * NKL];
        grad_bra_block<C, NAB>(U + C::G_U_F_LK * C::G_U_NE, C::G_U_NE,
                               [](const double *in, double *out, double x, double y, double z) {
                                   C::template hrr_im<double>(in, out, x, y, z);
                               }, br, kt, X);
        grad_bra_contract<C, 0, LI - 1, -1>(X, Wt, gA);
    }
    if constexpr (LJ > 0) {
        constexpr int NAB = NI * g_ncart(LJ - 1);
        double X[NAB * NKL];
        grad_bra_block<C, NAB>(U + C::G_U_F_LK * C::G_U_NE + C::G_U_E_LI, C::G_U_NE,
                               [](const double *in, double *out, double x, double y, double z) {
                                   C::template hrr_jm<double>(in, out, x, y, z);
                               }, br, kt, X);
        grad_bra_contract<C, 1, LJ - 1, -1>(X, Wt, gB);
    }
    if constexpr (LK > 0) {
        // U's f range is [lk - 1, lkl]; the lowered transfer reads [lk - 1, lkl - 1]
        constexpr int NFM = C::G_U_NF - g_ncart(LK + LL), NKS = g_ncart(LK - 1) * NL;
        double tb[NFM * NIJ];
#pragma unroll
        for (int f = 0; f < NFM; ++f)
            C::template hrr_bra<double>(U + f * C::G_U_NE + C::G_U_E_LI, tb + f * NIJ, br.ABx,
                                        br.ABy, br.ABz);
        double X[NIJ * NKS];
#pragma unroll
        for (int ij = 0; ij < NIJ; ++ij) {
            double row[NFM];
#pragma unroll
            for (int f = 0; f < NFM; ++f) row[f] = tb[f * NIJ + ij];
            C::template hrr_km<double>(row, X + ij * NKS, kt.ABx, kt.ABy, kt.ABz);
        }
        grad_ket_contract<C, LK - 1, -1>(X, Wt, gC);
    }
}

// RA: shell i raised
template <class C>
__device__ __forceinline__ void grad_from_ra(const double *RA, const double *Wt, const PairRec &br,
                                             const PairRec &kt, double gA[3])
{
    constexpr int NAB = g_ncart(C::LI + 1) * C::NJ, NKL = C::NK * C::NL;
    double X[NAB * NKL];
    grad_bra_block<C, NAB>(RA, C::G_RA_NE,
                           [](const double *in, double *out, double x, double y, double z) {
                               C::template hrr_ip<double>(in, out, x, y, z);
                           }, br, kt, X);
    grad_bra_contract<C, 0, C::LI + 1, 1>(X, Wt, gA);
}

// RB: shell j raised
template <class C>
__device__ __forceinline__ void grad_from_rb(const double *RB, const double *Wt, const PairRec &br,
                                             const PairRec &kt, double gB[3])
{
    constexpr int NAB = C::NI * g_ncart(C::LJ + 1), NKL = C::NK * C::NL;
    double X[NAB * NKL];
    grad_bra_block<C, NAB>(RB, C::G_RB_NE,
                           [](const double *in, double *out, double x, double y, double z) {
                               C::template hrr_jp<double>(in, out, x, y, z);
                           }, br, kt, X);
    grad_bra_contract<C, 1, C::LJ + 1, 1>(X, Wt, gB);
}

// RC: shell k raised (f levels lk + 1 ..)
template <class C>
__device__ __forceinline__ void grad_from_rc(const double *RC, const double *Wt, const PairRec &br,
                                             const PairRec &kt, double gC[3])
{
    constexpr int NIJ = C::NI * C::NJ;
    constexpr int NFS = C::G_RC_NF, NKS = g_ncart(C::LK + 1) * C::NL;
    double tb[NFS * NIJ];
#pragma unroll
    for (int f = 0; f < NFS; ++f)
        C::template hrr_bra<double>(RC + f * C::G_RC_NE, tb + f * NIJ, br.ABx, br.ABy, br.ABz);
    double X[NIJ * NKS];
#pragma unroll
    for (int ij = 0; ij < NIJ; ++ij) {
        double row[NFS];
#pragma unroll
        for (int f = 0; f < NFS; ++f) row[f] = tb[f * NIJ + ij];
        C::template hrr_kp<double>(row, X + ij * NKS, kt.ABx, kt.ABy, kt.ABz);
    }
    grad_ket_contract<C, C::LK + 1, 1>(X, Wt, gC);
}

template <class C>
__device__ __forceinline__ void grad_quartet(const ClassArgs &A, const PlanView &V,
                                             const PairRec &br, const double *__restrict__ sbra,
                                             int entry, double sym, double gb[6], double *fsum)
{
    constexpr int NIJ = C::NI * C::NJ, NKL = C::NK * C::NL;
    constexpr int NU = C::G_U_NE * C::G_U_NF, NRA = C::G_RA_NE * C::G_RA_NF;
    constexpr int NRB = C::G_RB_NE * C::G_RB_NF, NRC = C::G_RC_NE * C::G_RC_NF;
    const int kk = entry & JK_Q_KET;
    const PairRec kt = V.ket[kk];
    const double fac = kt.ish == kt.jsh ? 0.5 * sym : sym;
    double gA[3] = {0., 0., 0.}, gB[3] = {0., 0., 0.}, gC[3] = {0., 0., 0.};
    if constexpr (!C::G_SPLIT) {
        double U[NU], RA[NRA], RB[NRB], RC[NRC];
#pragma unroll
        for (int n = 0; n < NU; ++n) U[n] = 0.;
#pragma unroll
        for (int n = 0; n < NRA; ++n) RA[n] = 0.;
#pragma unroll
        for (int n = 0; n < NRB; ++n) RB[n] = 0.;
#pragma unroll
        for (int n = 0; n < NRC; ++n) RC[n] = 0.;
        grad_accum<C, -1>(A, V, br, kt, sbra, U, RA, RB, RC);
        double Wt[NIJ * NKL];
        grad_w<C>(A, V, br, kt, fac, Wt);
        grad_from_ra<C>(RA, Wt, br, kt, gA);
        grad_from_rb<C>(RB, Wt, br, kt, gB);
        grad_from_rc<C>(RC, Wt, br, kt, gC);
        grad_from_u<C>(U, Wt, br, kt, gA, gB, gC);
    } else {
        // one block per pass over the primitives; W re-formed for each
        // contraction (density loads, L1/L2 hits) rather than kept live
        // through the primitive loops
        {
            double U[NU];
#pragma unroll
            for (int n = 0; n < NU; ++n) U[n] = 0.;
            grad_accum<C, 0>(A, V, br, kt, sbra, U, nullptr, nullptr, nullptr);
            double Wt[NIJ * NKL];
            grad_w<C>(A, V, br, kt, fac, Wt);
            grad_from_u<C>(U, Wt, br, kt, gA, gB, gC);
        }
        {
            double RA[NRA];
#pragma unroll
            for (int n = 0; n < NRA; ++n) RA[n] = 0.;
            grad_accum<C, 1>(A, V, br, kt, sbra, nullptr, RA, nullptr, nullptr);
            double Wt[NIJ * NKL];
            grad_w<C>(A, V, br, kt, fac, Wt);
            grad_from_ra<C>(RA, Wt, br, kt, gA);
        }
        {
            double RB[NRB];
#pragma unroll
            for (int n = 0; n < NRB; ++n) RB[n] = 0.;
            grad_accum<C, 2>(A, V, br, kt, sbra, nullptr, nullptr, RB, nullptr);
            double Wt[NIJ * NKL];
            grad_w<C>(A, V, br, kt, fac, Wt);
            grad_from_rb<C>(RB, Wt, br, kt, gB);
        }
        {
            double RC[NRC];
#pragma unroll
            for (int n = 0; n < NRC; ++n) RC[n] = 0.;
            grad_accum<C, 3>(A, V, br, kt, sbra, nullptr, nullptr, nullptr, RC);
            double Wt[NIJ * NKL];
            grad_w<C>(A, V, br, kt, fac, Wt);
            grad_from_rc<C>(RC, Wt, br, kt, gC);
        }
    }
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        gb[x] += gA[x];
        gb[3 + x] += gB[x];
    }
    // ket atoms: shell k, and shell l by translational invariance
    const int ak = A.sh_atom[kt.ish], al = A.sh_atom[kt.jsh];
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        atomicAdd(fsum + ak * 3 + x, gC[x]);
        atomicAdd(fsum + al * 3 + x, -(gA[x] + gB[x] + gC[x]));
    }
}

// ---------------------------------------------------------------------------
// team form (the classes whose blocks do not fit one lane): a warp per
// quartet.  Per primitive quartet, lane (root, direction) builds that root's
// 2D integrals with both transfers applied, g[i][j][k][l] for i <= li + 1,
// j <= lj + 1, k <= lk + 1, l <= ll (the corners no derivative reads are
// left out), into shared memory; every lane then takes a strided share of
// the class's (a, b, c, d) components and adds W_abcd times the derivative
// integrals of shells i, j, k.  W is formed once per quartet in shared
// memory.
template <class C>
struct GradTeam {
    static constexpr int LI = C::LI, LJ = C::LJ, LK = C::LK, LL = C::LL;
    static constexpr int NR = C::G_NROOTS;
    static constexpr int NIJKL = C::NI * C::NJ * C::NK * C::NL;
    static constexpr int SK = LL + 1, SJ = (LK + 2) * SK, SI = (LJ + 2) * SJ;
    // one root and direction, padded to an odd count so that the 3 NR lanes
    // writing their tables at the same offsets hit different banks
    static constexpr int GS = ((LI + 2) * SI) | 1;
    static constexpr int W = 0, RW = NIJKL, G = (RW + 2 * NR + 1) & ~1;
    static constexpr int SIZE = G + 3 * NR * GS;             // doubles per warp
    // warps per block: as many as fit in about 150 KB beside the bra records
    static constexpr int NW0 = 150000 / (SIZE * 8 + 4096);
    static constexpr int NW = NW0 < 1 ? 1 : (NW0 > 4 ? 4 : NW0);
};

// one root and direction: the 2D integrals V[e][f] (e <= lij + 1, f <= lkl + 1)
// by the recurrences, then the bra transfer (a, b + 1) = (a + 1, b) + AB (a, b)
// level by level in place and, for each (i, j) row kept, the ket transfer the
// same way; out[((i * (lj + 2) + j) * (lk + 2) + k) * (ll + 1) + l]
template <class C>
__device__ __forceinline__ void grad_team_table(double c0, double cp, double b00, double b10, double b01,
                                             double g00, double ab, double cd, double *out)
{
    using T = GradTeam<C>;
    constexpr int E1 = C::LIJ + 1, F1 = C::LKL + 1, FW = F1 + 1;
    double v[(E1 + 1) * FW];
    v[0] = g00;
    v[FW] = c0 * g00;
#pragma unroll
    for (int e = 1; e < E1; ++e) v[(e + 1) * FW] = fma(e * b10, v[(e - 1) * FW], c0 * v[e * FW]);
#pragma unroll
    for (int f = 0; f < F1; ++f) {
        v[f + 1] = f ? fma(f * b01, v[f - 1], cp * v[f]) : cp * v[f];
#pragma unroll
        for (int e = 1; e <= E1; ++e) {
            double t = fma(e * b00, v[(e - 1) * FW + f], cp * v[e * FW + f]);
            if (f) t = fma(f * b01, v[e * FW + f - 1], t);
            v[e * FW + f + 1] = t;
        }
    }
#pragma unroll
    for (int j = 0; j <= T::LJ + 1; ++j) {
        if (j) {   // level j from level j - 1: rows i <= E1 - j
#pragma unroll
            for (int i = 0; i <= E1 - j; ++i)
#pragma unroll
                for (int f = 0; f < FW; ++f) v[i * FW + f] = fma(ab, v[i * FW + f], v[(i + 1) * FW + f]);
        }
        const int imax = T::LI + 1 < E1 - j ? T::LI + 1 : E1 - j;
#pragma unroll
        for (int i = 0; i <= imax; ++i) {
            double r[FW];
#pragma unroll
            for (int f = 0; f < FW; ++f) r[f] = v[i * FW + f];
            double *o = out + i * T::SI + j * T::SJ;
#pragma unroll
            for (int l = 0; l <= T::LL; ++l) {
                if (l) {
#pragma unroll
                    for (int k = 0; k <= F1 - l; ++k) r[k] = fma(cd, r[k], r[k + 1]);
                }
                const int kmax = T::LK + 1 < F1 - l ? T::LK + 1 : F1 - l;
#pragma unroll
                for (int k = 0; k <= kmax; ++k) o[k * T::SK + l] = r[k];
            }
        }
    }
}

template <class C>
__device__ __forceinline__ void grad_team_quartet(const ClassArgs &A, const PlanView &V,
                                                  const PairRec &br, const double *__restrict__ sbra,
                                                  int entry, double sym, double *ws, int lane,
                                                  double *fsum)
{
    using T = GradTeam<C>;
    constexpr int NR = T::NR, NJ = C::NJ, NK = C::NK, NL = C::NL, NKL = NK * NL;
    const int kk = entry & JK_Q_KET;
    const PairRec kt = V.ket[kk];
    double *Wq = ws + T::W, *rw = ws + T::RW, *G = ws + T::G;
    const double fac = kt.ish == kt.jsh ? 0.5 * sym : sym;
    const size_t nao = V.nao, nao2 = nao * nao;
    __syncwarp();   // the previous quartet's readers are done with W and G
    for (int e = lane; e < T::NIJKL; e += 32) {
        const int a = e / (NJ * NKL), b = (e / NKL) % NJ, c = (e / NL) % NK, d = e % NL;
        const size_t ia = br.i0 + a, jb = br.j0 + b, kc = kt.i0 + c, ld = kt.j0 + d;
        double dab = 0., dcd = 0.;
        for (int s = 0; s < V.n_j; ++s) {
            const double *ds = V.dsJ + s * nao2;
            dab += __ldg(ds + ia * nao + jb);
            dcd += __ldg(ds + kc * nao + ld);
        }
        double w = 0.25 * A.grad_wj * dab * dcd;
        for (int s = 0; s < V.n_k; ++s) {
            const double *D = V.dmK + s * nao2;
            w -= A.grad_wk * fma(__ldg(D + ia * nao + kc), __ldg(D + jb * nao + ld),
                                 __ldg(D + ia * nao + ld) * __ldg(D + jb * nao + kc));
        }
        Wq[e] = fac * w;
    }
    double gA[3] = {0., 0., 0.}, gB[3] = {0., 0., 0.}, gC[3] = {0., 0., 0.};
    const double io2 = A.op_inv_om2[0];
    const double AB[3] = {br.ABx, br.ABy, br.ABz}, CD[3] = {kt.ABx, kt.ABy, kt.ABz};
    for (int kp = 0; kp < kt.nprim; ++kp) {
        const double *kr = V.prim + (size_t)(kt.prim0 + kp) * JK_PRIM_STRIDE;
        const double akl = __ldg(kr + PR_A), hiq = __ldg(kr + PR_HIA), kq = __ldg(kr + PR_KP);
        const double wC = 2.0 * __ldg(kr + PR_AI);
        for (int bp = 0; bp < br.nprim; ++bp) {
            const double *s = sbra + bp * JK_PRIM_STRIDE;
            const double aij = s[PR_A], hip = s[PR_HIA];
            const double wA = 2.0 * s[PR_AI], wB = 2.0 * (aij - s[PR_AI]);
            const double PQ[3] = {s[PR_PX] - __ldg(kr + PR_PX), s[PR_PX + 1] - __ldg(kr + PR_PX + 1),
                                  s[PR_PX + 2] - __ldg(kr + PR_PX + 2)};
            const double rs = rsqrt(fma(aij * akl, io2, aij + akl));
            const double is = rs * rs;
            const double x = aij * akl * is * fma(PQ[0], PQ[0], fma(PQ[1], PQ[1], PQ[2] * PQ[2]));
            __syncwarp();   // G of the previous primitive quartet is read
            if (lane < 2 * NR) rw[lane] = rys_row<NR>(x, A.rys, lane);
            __syncwarp();
            if (lane < 3 * NR) {
                const int r = lane / 3, d = lane - 3 * (lane / 3);
                const double uis = rw[r] * is;
                const double up = uis * akl, uq = uis * aij;
                const double g00 = d == 2 ? rw[NR + r] * s[PR_KP] * kq * rs : 1.0;
                grad_team_table<C>(fma(-up, PQ[d], s[PR_PAX + d]), fma(uq, PQ[d], __ldg(kr + PR_PAX + d)),
                                   0.5 * uis, fma(-hip, up, hip), fma(-hiq, uq, hiq), g00, AB[d],
                                   CD[d], G + (r * 3 + d) * T::GS);
            }
            __syncwarp();
            for (int e = lane; e < T::NIJKL; e += 32) {
                const int a = e / (NJ * NKL), b = (e / NKL) % NJ, c = (e / NL) % NK, d = e % NL;
                int pw[4][3], off[3];
#pragma unroll
                for (int x3 = 0; x3 < 3; ++x3) {
                    pw[0][x3] = g_comp(C::LI, a, x3);
                    pw[1][x3] = g_comp(C::LJ, b, x3);
                    pw[2][x3] = g_comp(C::LK, c, x3);
                    pw[3][x3] = g_comp(C::LL, d, x3);
                    off[x3] = pw[0][x3] * T::SI + pw[1][x3] * T::SJ + pw[2][x3] * T::SK + pw[3][x3];
                }
                double tA[3] = {0., 0., 0.}, tB[3] = {0., 0., 0.}, tC[3] = {0., 0., 0.};
#pragma unroll 1
                for (int r = 0; r < NR; ++r) {
                    const double *g3[3] = {G + (r * 3) * T::GS + off[0], G + (r * 3 + 1) * T::GS + off[1],
                                           G + (r * 3 + 2) * T::GS + off[2]};
                    const double g0[3] = {g3[0][0], g3[1][0], g3[2][0]};
#pragma unroll
                    for (int x3 = 0; x3 < 3; ++x3) {
                        const double *q = g3[x3];
                        const double o2 = g0[(x3 + 1) % 3] * g0[(x3 + 2) % 3];
                        const int ia = pw[0][x3], jb = pw[1][x3], kc = pw[2][x3];
                        double dA = wA * q[T::SI], dB = wB * q[T::SJ], dC = wC * q[T::SK];
                        if (ia) dA = fma(-(double)ia, q[-T::SI], dA);
                        if (jb) dB = fma(-(double)jb, q[-T::SJ], dB);
                        if (kc) dC = fma(-(double)kc, q[-T::SK], dC);
                        tA[x3] = fma(dA, o2, tA[x3]);
                        tB[x3] = fma(dB, o2, tB[x3]);
                        tC[x3] = fma(dC, o2, tC[x3]);
                    }
                }
                const double w = Wq[e];
#pragma unroll
                for (int x3 = 0; x3 < 3; ++x3) {
                    gA[x3] = fma(w, tA[x3], gA[x3]);
                    gB[x3] = fma(w, tB[x3], gB[x3]);
                    gC[x3] = fma(w, tC[x3], gC[x3]);
                }
            }
        }
    }
    double g9[9] = {gA[0], gA[1], gA[2], gB[0], gB[1], gB[2], gC[0], gC[1], gC[2]};
#pragma unroll
    for (int c = 0; c < 9; ++c) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) g9[c] += __shfl_xor_sync(0xffffffffu, g9[c], o);
    }
    if (lane == 0) {
        const int at[3] = {A.sh_atom[br.ish], A.sh_atom[br.jsh], A.sh_atom[kt.ish]};
        const int al = A.sh_atom[kt.jsh];
#pragma unroll
        for (int x3 = 0; x3 < 3; ++x3) {
            atomicAdd(fsum + at[0] * 3 + x3, g9[x3]);
            atomicAdd(fsum + at[1] * 3 + x3, g9[3 + x3]);
            atomicAdd(fsum + at[2] * 3 + x3, g9[6 + x3]);
            atomicAdd(fsum + al * 3 + x3, -(g9[x3] + g9[3 + x3] + g9[6 + x3]));
        }
    }
}

// one task: bra pair task.bra against kets [task.k0, task.k1)
template <class C>
__device__ __forceinline__ void grad_task(const ClassArgs &A, const PlanView &V, const Task &task,
                                          RegWarp &w, double *ws, int lane, double *fsum)
{
    const int b = task.bra;
    const PairRec br = V.bra[b];
    if (b != w.staged_b || task.view != w.staged_v) {
        __syncwarp();
        const double *src = V.prim + (size_t)br.prim0 * JK_PRIM_STRIDE;
        for (int t = lane; t < br.nprim * JK_PRIM_STRIDE; t += 32) w.sbra[t] = src[t];
        __syncwarp();
        w.staged_b = b;
        w.staged_v = task.view;
    }
    const double sym_b = br.ish == br.jsh ? 0.5 : 1.0;
    const bool diag = V.same_class;
    double gb[6] = {0., 0., 0., 0., 0., 0.};
    int *q = w.q;
    int nq = 0;
    auto run = [&](int n) {
        if constexpr (C::G_SMALL) {
            if (lane < n) {
                const int e2 = q[lane], k2 = e2 & JK_Q_KET;
                grad_quartet<C>(A, V, br, w.sbra, e2, diag && k2 == b ? 0.5 * sym_b : sym_b, gb, fsum);
                w.npq += (unsigned long long)br.nprim * V.ket[k2].nprim;
            }
        } else {
            for (int t = 0; t < n; ++t) {
                const int e2 = q[t], k2 = e2 & JK_Q_KET;
                grad_team_quartet<C>(A, V, br, w.sbra, e2, diag && k2 == b ? 0.5 * sym_b : sym_b,
                                     ws, lane, fsum);
                if (lane == 0) w.npq += (unsigned long long)br.nprim * V.ket[k2].nprim;
            }
        }
        w.nq += n;
        __syncwarp();
    };
    for (int base = task.k0; base < task.k1; base += 32) {
        const int kk = base + lane;
        float bK = JK_NEG_INF, bJ = JK_NEG_INF;
        if (kk < task.k1) quartet_bounds(V, br.ish, br.jsh, br.q, V.ket + kk, bK, bJ);
        // a quartet counts when its Coulomb or exchange bound passes: the
        // gradient takes both terms of every quartet it evaluates
        const bool keep = fmaxf(bK, bJ) > V.log_tol;
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) q[nq + __popc(m & ((1u << lane) - 1u))] = kk;
        nq += __popc(m);
        __syncwarp();
        if (nq >= 32) {
            run(32);
            if (lane < nq - 32) q[lane] = q[32 + lane];
            __syncwarp();
            nq -= 32;
        }
    }
    if (nq) run(nq);
    // bra atoms: one atomic per component and task
    const int ai = A.sh_atom[br.ish], aj = A.sh_atom[br.jsh];
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        double v = gb[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) atomicAdd(fsum + (c < 3 ? ai : aj) * 3 + c % 3, v);
    }
}

// per-lane form (G_SMALL classes): 4 warps of quartets; team form: a warp
// per quartet, GradTeam<C>::NW warps with their shared workspaces
template <class C>
constexpr int grad_threads() { return C::G_SMALL ? 128 : 32 * GradTeam<C>::NW; }

template <class C>
constexpr size_t grad_team_doubles() { return C::G_SMALL ? 0 : (size_t)GradTeam<C>::SIZE; }

// resident blocks per SM the gradient kernels are compiled for, measured
// per class on (H2O)_32 6-31G* and (H2O)_16 def2-TZVP UHF: the per-lane
// kernels of (ss|ss) and (ps|ss) at 4 (128 registers; (ps|ss) 10.6 -> 9.6
// ms, while (ps|ps) and (ds|ss) spill at that cap and lose, 4.2 -> 7.6 and
// 3.9 -> 6.0 ms), the other per-lane kernels at 1 (255 registers); the
// per-warp kernels at 3 (at most 170 registers; shared memory allows 3:
// (dp|ds) 10.2 -> 8.8 ms, (dd|ps) 8.3 -> 7.5, (dp|pp) 8.2 -> 7.6), except
// (pp|pp), (dp|dp), (fp|ps), (fp|pp), which lose at 3 (7.2 -> 7.9, 6.8 ->
// 8.2, 38.0 -> 43.7, 59.7 -> 70.5 ms) and keep 1
template <class C>
constexpr int grad_min_blocks()
{
    constexpr int tag = ((C::LI * 10 + C::LJ) * 10 + C::LK) * 10 + C::LL;
    if constexpr (C::G_SMALL) return !C::G_SPLIT && C::G_NMEM <= 20 ? 4 : 1;
    return tag == 1111 || tag == 2121 || tag == 3110 || tag == 3111 ? 1 : 3;
}

template <class C, int NT>
__global__ void __launch_bounds__(NT, grad_min_blocks<C>())
    jk_grad_kernel(const __grid_constant__ LaunchParams<1> P)
{
    const ClassArgs &A = P.a;
    constexpr int NW = NT / 32;
    extern __shared__ double smem[];
    __shared__ int s_q[NW][64];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    RegWarp w;
    w.sbra = smem + warp * A.max_bra_prim * JK_PRIM_STRIDE;
    double *ws = smem + NW * A.max_bra_prim * JK_PRIM_STRIDE + warp * grad_team_doubles<C>();
    // forces: summed per block in shared memory when the atoms fit, else
    // straight to the output
    const bool fsmem = A.natm <= JK_GRAD_SMEM_ATOMS;
    double *fsum = fsmem ? smem + NW * (A.max_bra_prim * JK_PRIM_STRIDE + grad_team_doubles<C>())
                         : A.grad;
    if (fsmem) {
        for (int t = threadIdx.x; t < 3 * A.natm; t += NT) fsum[t] = 0.;
        __syncthreads();
    }
    w.sbra32 = nullptr;
    w.q = s_q[warp];
    w.staged_v = w.staged_b = -1;
    w.nq = w.npq = w.nq32 = 0;
    int t_begin, t_end;
    launch_tasks(A, t_begin, t_end);
    const int chunk = *A.chunk;
    Task task;
    while (claim_task(P, t_begin, t_end, chunk, task)) grad_task<C>(A, P.v[0], task, w, ws, lane, fsum);
    if (fsmem) {
        __syncthreads();
        for (int t = threadIdx.x; t < 3 * A.natm; t += NT)
            if (fsum[t] != 0.) atomicAdd(A.grad + t, fsum[t]);
    }
    if (lane == 0 && A.nquartets) atomicAdd(A.nquartets, w.nq);
    unsigned long long npq = w.npq;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) npq += __shfl_down_sync(0xffffffffu, npq, o);
    if (lane == 0 && A.nprimq && npq) atomicAdd(A.nprimq, npq);
}

template <class C>
static int launch_grad(const ClassArgs &a, const PlanView *views, const LaunchCfg &cfg,
                       const char *tag, KernelState &ks)
{
    constexpr int NT = grad_threads<C>();
    static LaunchParams<1> prm;
    prm.a = a;
    prm.v[0] = views[0];
    auto kern = jk_grad_kernel<C, NT>;
    const size_t shm =
        ((size_t)(NT / 32) * (a.max_bra_prim * JK_PRIM_STRIDE + grad_team_doubles<C>()) +
         (a.natm <= JK_GRAD_SMEM_ATOMS ? 3 * (size_t)a.natm : 0)) * sizeof(double);
    int bps = 0;
    const int rc = configure(kern, NT, shm, ks, cfg, tag, bps);
    if (rc || cfg.configure_only) return rc;
    const int grid = cfg.num_sms * bps;
    kern<<<grid, NT, shm, cfg.stream>>>(prm);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess && cfg.msg)
        snprintf(cfg.msg, 256, "class %s gradient: launch of %d x %d threads, %zu B shared: %s", tag,
                 grid, NT, shm, cudaGetErrorString(e));
    return (int)e;
}
