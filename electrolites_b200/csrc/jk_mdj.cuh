// McMurchie-Davidson J (J-only builds), register form, one quartet per lane.
//
// The reference's J engine (electrolites/fastj.py:540-569, kernels from
// electrolites/codegen/gen_j_high.py; GPU4PySCF's MD_build_j) expands every
// primitive pair in Hermite Gaussians: with E^{ab}_{tuv} the Hermite
// coefficients of the Cartesian pair (a on A, b on B, exponent sum p),
//   (ab|cd) = sum_{pq} K_p K_q / sqrt(p+q) sum_{tuv} E^{ab}_{tuv}(p)
//             sum_{tau nu phi} (-1)^{tau+nu+phi} E^{cd}_{tau nu phi}(q)
//             R_{t+tau, u+nu, v+phi}(alpha, P - Q),
// R^{(n)}_{000} = (-2 alpha)^n F_n(alpha |PQ|^2), alpha = p q / (p + q),
// R^{(n)}_{t+1,u,v} = t R^{(n+1)}_{t-1,u,v} + X_PQ R^{(n+1)}_{t,u,v} (and the
// same in u with Y, v with Z), K_p = sqrt(2 pi^{5/2}) K_ab / p the pair's
// record prefactor.  The J digest of a unique quartet, the same as the Rys
// forms' (J_h(Q)[cd] += fac sum_ab (ab|cd) Ds[ab], J_h(P)[ab] += fac sum_cd
// (ab|cd) Ds[cd], Ds = D + D^T), then runs through the Hermite densities
//   D^_p[tuv] = K_p sum_ab E^{ab}_{tuv}(p) Ds[ab]:
// ket side J^_q[tnf] += (-1)^{t+n+f} sum_{tuv} D^_p[tuv] R_{...} summed over
// the bra primitives, then J_h(Q)[cd] += K_q sum E^{cd}(q) J^_q; bra side
// j^_p[tuv] = sum_{tnf} (-1)^{t+n+f} D^_q[tnf] R_{...}, J_h(P)[ab] +=
// K_p sum E^{ab}(p) j^_p per primitive quartet, summed over the task in
// registers.
//
// The Boys values come from the class's Rys quadrature, which integrates
// t^{2n} exactly for n <= 2 NROOTS - 1 >= L: F_n(T) = sum_r w_r u_r^n with
// u_r = t_r^2 the roots and w_r the weights (summing to F_0).
//
// The bra pair's Hermite densities are formed once per task by the warp
// (shared memory, JK_MD_DENS densities); the ket's per primitive in the lane.
#pragma once

__host__ __device__ constexpr int md_nt(int L) { return L < 0 ? 0 : (L + 1) * (L + 2) * (L + 3) / 6; }

// index of Hermite (t, u, v): by level s = t + u + v, then (u + v, v)
__host__ __device__ constexpr int md_h(int t, int u, int v)
{
    return md_nt(t + u + v - 1) + (u + v) * (u + v + 1) / 2 + v;
}

template <class C>
constexpr bool md_class()
{
    return C::REG && C::LI + C::LJ + C::LK + C::LL <= JK_MD_LMAX;
}

// E^{ab}_t of one direction for a <= LA, b <= LB, at [(a * (LB + 1) + b) *
// (LA + LB + 1) + t]: E^{a+1,b}_t = hp E^{ab}_{t-1} + pa E^{ab}_t +
// (t + 1) E^{ab}_{t+1}, and in b with pb; hp = 1 / (2 p), pa = P - A, pb = P - B
template <int LA, int LB>
__device__ __forceinline__ void md_e(double pa, double pb, double hp,
                                     double E[(LA + 1) * (LB + 1) * (LA + LB + 1)])
{
    constexpr int W = LA + LB + 1;
#pragma unroll
    for (int n = 0; n < (LA + 1) * (LB + 1) * W; ++n) E[n] = 0.;
    E[0] = 1.;
#pragma unroll
    for (int a = 1; a <= LA; ++a)
#pragma unroll
        for (int t = 0; t <= a; ++t) {
            const int o = ((a - 1) * (LB + 1)) * W;
            double s = pa * E[o + t];
            if (t > 0) s = fma(hp, E[o + t - 1], s);
            if (t + 1 <= a - 1) s = fma(double(t + 1), E[o + t + 1], s);
            E[(a * (LB + 1)) * W + t] = s;
        }
#pragma unroll
    for (int b = 1; b <= LB; ++b)
#pragma unroll
        for (int a = 0; a <= LA; ++a)
#pragma unroll
            for (int t = 0; t <= a + b; ++t) {
                const int o = (a * (LB + 1) + b - 1) * W;
                double s = t <= a + b - 1 ? pb * E[o + t] : 0.;
                if (t > 0) s = fma(hp, E[o + t - 1], s);
                if (t + 1 <= a + b - 1) s = fma(double(t + 1), E[o + t + 1], s);
                E[(a * (LB + 1) + b) * W + t] = s;
            }
}

// D^[tuv] = kp sum_ab blk[a * NB + b] Ex Ey Ez over the pair's Cartesian
// components (PySCF order)
template <int LA, int LB>
__device__ __forceinline__ void md_dhat(const double *Ex, const double *Ey, const double *Ez,
                                        const double *blk, double kp, double *dh)
{
    constexpr int NA = (LA + 1) * (LA + 2) / 2, NB = (LB + 1) * (LB + 2) / 2, W = LA + LB + 1;
#pragma unroll
    for (int h = 0; h < md_nt(LA + LB); ++h) dh[h] = 0.;
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int ax = g_comp(LA, a, 0), ay = g_comp(LA, a, 1), az = g_comp(LA, a, 2);
            const int bx = g_comp(LB, b, 0), by = g_comp(LB, b, 1), bz = g_comp(LB, b, 2);
            const double d = blk[a * NB + b] * kp;
#pragma unroll
            for (int t = 0; t <= ax + bx; ++t) {
                const double ex = d * Ex[(ax * (LB + 1) + bx) * W + t];
#pragma unroll
                for (int u = 0; u <= ay + by; ++u) {
                    const double exy = ex * Ey[(ay * (LB + 1) + by) * W + u];
#pragma unroll
                    for (int v = 0; v <= az + bz; ++v)
                        dh[md_h(t, u, v)] = fma(exy, Ez[(az * (LB + 1) + bz) * W + v], dh[md_h(t, u, v)]);
                }
            }
        }
}

// out[a * NB + b] += kp sum_tuv Ex Ey Ez jh[tuv]
template <int LA, int LB>
__device__ __forceinline__ void md_back(const double *Ex, const double *Ey, const double *Ez,
                                        const double *jh, double kp, double *out)
{
    constexpr int NA = (LA + 1) * (LA + 2) / 2, NB = (LB + 1) * (LB + 2) / 2, W = LA + LB + 1;
#pragma unroll
    for (int a = 0; a < NA; ++a)
#pragma unroll
        for (int b = 0; b < NB; ++b) {
            const int ax = g_comp(LA, a, 0), ay = g_comp(LA, a, 1), az = g_comp(LA, a, 2);
            const int bx = g_comp(LB, b, 0), by = g_comp(LB, b, 1), bz = g_comp(LB, b, 2);
            double s = 0.;
#pragma unroll
            for (int t = 0; t <= ax + bx; ++t) {
                const double ex = Ex[(ax * (LB + 1) + bx) * W + t];
#pragma unroll
                for (int u = 0; u <= ay + by; ++u) {
                    const double exy = ex * Ey[(ay * (LB + 1) + by) * W + u];
#pragma unroll
                    for (int v = 0; v <= az + bz; ++v)
                        s = fma(exy * Ez[(az * (LB + 1) + bz) * W + v], jh[md_h(t, u, v)], s);
                }
            }
            out[a * NB + b] = fma(kp, s, out[a * NB + b]);
        }
}

// R_{tuv} (t + u + v <= L) from Fn[n] = R^{(n)}_{000}, n = 0..L
template <int L>
__device__ __forceinline__ void md_r(const double *Fn, double X, double Y, double Z, double *R)
{
    constexpr int NT = md_nt(L);
    double P[NT];
    P[0] = Fn[L];
#pragma unroll
    for (int n = L - 1; n >= 0; --n) {
        double Q[NT];
#pragma unroll
        for (int s = 0; s <= L - n; ++s)
#pragma unroll
            for (int a = 0; a <= s; ++a)
#pragma unroll
                for (int v = 0; v <= a; ++v) {
                    const int u = a - v, t = s - a;
                    double r;
                    if (s == 0) {
                        r = Fn[n];
                    } else if (t > 0) {
                        r = X * P[md_h(t - 1, u, v)];
                        if (t > 1) r = fma(double(t - 1), P[md_h(t - 2, u, v)], r);
                    } else if (u > 0) {
                        r = Y * P[md_h(t, u - 1, v)];
                        if (u > 1) r = fma(double(u - 1), P[md_h(t, u - 2, v)], r);
                    } else {
                        r = Z * P[md_h(t, u, v - 1)];
                        if (v > 1) r = fma(double(v - 1), P[md_h(t, u, v - 2)], r);
                    }
                    Q[md_h(t, u, v)] = r;
                }
#pragma unroll
        for (int h = 0; h < md_nt(L - n); ++h) P[h] = Q[h];
    }
#pragma unroll
    for (int h = 0; h < NT; ++h) R[h] = P[h];
}

// the bra pair's Hermite densities of one primitive and density into dh
template <class C>
__device__ __forceinline__ void md_bra_dens(const PlanView &V, const PairRec &br,
                                            const double *s, int d, double *dh)
{
    constexpr int LI = C::LI, LJ = C::LJ, NI = C::NI, NJ = C::NJ, W = LI + LJ + 1;
    const size_t nao = V.nao;
    const double *ds = V.dsJ + (size_t)d * nao * nao;
    double blk[NI * NJ];
#pragma unroll
    for (int a = 0; a < NI; ++a)
#pragma unroll
        for (int b = 0; b < NJ; ++b) blk[a * NJ + b] = __ldg(ds + (br.i0 + a) * nao + br.j0 + b);
    double Ex[(LI + 1) * (LJ + 1) * W], Ey[(LI + 1) * (LJ + 1) * W], Ez[(LI + 1) * (LJ + 1) * W];
    const double hp = s[PR_HIA];
    md_e<LI, LJ>(s[PR_PAX], s[PR_PAX] + br.ABx, hp, Ex);
    md_e<LI, LJ>(s[PR_PAX + 1], s[PR_PAX + 1] + br.ABy, hp, Ey);
    md_e<LI, LJ>(s[PR_PAX + 2], s[PR_PAX + 2] + br.ABz, hp, Ez);
    md_dhat<LI, LJ>(Ex, Ey, Ez, blk, s[PR_KP], dh);
}

// one quartet: ket side into the ket pair's J_h block (atomics), bra side
// into jb[d * NIJ + ab] (the task's register sums); sdh: the bra's Hermite
// densities, [bp][d][md_nt(l_i + l_j)]
template <class C, bool SMEM>
__device__ __forceinline__ void md_quartet(const ClassArgs &A, const PlanView &V,
                                           const PairRec &br, const double *__restrict__ sbra,
                                           const double *__restrict__ sdh, int entry, double sym,
                                           const double *__restrict__ cheb, double *jb)
{
    constexpr int LI = C::LI, LJ = C::LJ, LK = C::LK, LL = C::LL;
    constexpr int LP = LI + LJ, LQ = LK + LL, L = LP + LQ;
    constexpr int NTP = md_nt(LP), NTQ = md_nt(LQ), NIJ = C::NI * C::NJ;
    constexpr int NK = C::NK, NL = C::NL, NKL = NK * NL, N = C::NROOTS;
    constexpr int WP = LP + 1, WQ = LQ + 1;
    const int kk = entry & JK_Q_KET;
    const PairRec kt = V.ket[kk];
    const int n_j = V.n_j;
    const double fac = kt.ish == kt.jsh ? 0.5 * sym : sym;
    const size_t nao = V.nao, nao2 = nao * nao;
    double dkl[JK_MD_DENS][NKL], jkl[JK_MD_DENS][NKL];
#pragma unroll
    for (int d = 0; d < JK_MD_DENS; ++d)
#pragma unroll
        for (int c = 0; c < NK; ++c)
#pragma unroll
            for (int e = 0; e < NL; ++e) {
                dkl[d][c * NL + e] = d < n_j ? __ldg(V.dsJ + d * nao2 + (kt.i0 + c) * nao + kt.j0 + e) : 0.;
                jkl[d][c * NL + e] = 0.;
            }
    const double *ks = V.prim_soa + kt.soa;
    const size_t sn = (size_t)kt.soa_n;
    for (int kp = 0; kp < kt.nprim; ++kp) {
        const double *kr = ks + (size_t)kp * JK_SOA_FIELDS * sn;
        const double akl = __ldg(kr + PR_A * sn), hiq = __ldg(kr + PR_HIA * sn);
        const double kq = __ldg(kr + PR_KP * sn);
        const double Qx = __ldg(kr + PR_PX * sn), Qy = __ldg(kr + (PR_PX + 1) * sn);
        const double Qz = __ldg(kr + (PR_PX + 2) * sn);
        const double QCx = __ldg(kr + PR_PAX * sn), QCy = __ldg(kr + (PR_PAX + 1) * sn);
        const double QCz = __ldg(kr + (PR_PAX + 2) * sn);
        double Kx[(LK + 1) * (LL + 1) * WQ], Ky[(LK + 1) * (LL + 1) * WQ], Kz[(LK + 1) * (LL + 1) * WQ];
        md_e<LK, LL>(QCx, QCx + kt.ABx, hiq, Kx);
        md_e<LK, LL>(QCy, QCy + kt.ABy, hiq, Ky);
        md_e<LK, LL>(QCz, QCz + kt.ABz, hiq, Kz);
        double dq[JK_MD_DENS][NTQ], jq[JK_MD_DENS][NTQ];
#pragma unroll
        for (int d = 0; d < JK_MD_DENS; ++d) {
            md_dhat<LK, LL>(Kx, Ky, Kz, dkl[d], kq, dq[d]);
#pragma unroll
            for (int h = 0; h < NTQ; ++h) jq[d][h] = 0.;
        }
        for (int bp = 0; bp < br.nprim; ++bp) {
            const double *s = sbra + bp * JK_PRIM_STRIDE;
            const double aij = s[PR_A];
            const double PQx = s[PR_PX] - Qx, PQy = s[PR_PX + 1] - Qy, PQz = s[PR_PX + 2] - Qz;
            const double rs = rsqrt(aij + akl);
            const double al = aij * akl * rs * rs;
            const double x = al * fma(PQx, PQx, fma(PQy, PQy, PQz * PQz));
            double r[N], w[N];
            rys_eval<N, SMEM>(x, cheb, A.rys, r, w);
            double Fn[L + 1];
            {
                double m2a = rs;   // (-2 alpha)^n rs
#pragma unroll
                for (int n = 0; n <= L; ++n) {
                    double f = 0.;
#pragma unroll
                    for (int q = 0; q < N; ++q) {
                        double un = w[q];
#pragma unroll
                        for (int e = 0; e < n; ++e) un *= r[q];
                        f += un;
                    }
                    Fn[n] = m2a * f;
                    m2a *= -2.0 * al;
                }
            }
            double R[md_nt(L)];
            md_r<L>(Fn, PQx, PQy, PQz, R);
            const double *dp = sdh + bp * (JK_MD_DENS * NTP);
            double Ax[(LI + 1) * (LJ + 1) * WP], Ay[(LI + 1) * (LJ + 1) * WP], Az[(LI + 1) * (LJ + 1) * WP];
            const double hip = s[PR_HIA];
            md_e<LI, LJ>(s[PR_PAX], s[PR_PAX] + br.ABx, hip, Ax);
            md_e<LI, LJ>(s[PR_PAX + 1], s[PR_PAX + 1] + br.ABy, hip, Ay);
            md_e<LI, LJ>(s[PR_PAX + 2], s[PR_PAX + 2] + br.ABz, hip, Az);
#pragma unroll
            for (int d = 0; d < JK_MD_DENS; ++d) {
                if (d >= n_j) break;
                double jp[NTP];
#pragma unroll
                for (int s1 = 0; s1 <= LP; ++s1)
#pragma unroll
                    for (int a1 = 0; a1 <= s1; ++a1)
#pragma unroll
                        for (int v1 = 0; v1 <= a1; ++v1) {
                            const int u1 = a1 - v1, t1 = s1 - a1, h1 = md_h(t1, u1, v1);
                            const double dph = dp[d * NTP + h1];
                            double sb = 0.;
#pragma unroll
                            for (int s2 = 0; s2 <= LQ; ++s2)
#pragma unroll
                                for (int a2 = 0; a2 <= s2; ++a2)
#pragma unroll
                                    for (int v2 = 0; v2 <= a2; ++v2) {
                                        const int u2 = a2 - v2, t2 = s2 - a2, h2 = md_h(t2, u2, v2);
                                        const double rv = R[md_h(t1 + t2, u1 + u2, v1 + v2)];
                                        const double sg = (s2 & 1) ? -rv : rv;
                                        jq[d][h2] = fma(sg, dph, jq[d][h2]);
                                        sb = fma(sg, dq[d][h2], sb);
                                    }
                            jp[h1] = sb;
                        }
                md_back<LI, LJ>(Ax, Ay, Az, jp, fac * s[PR_KP], jb + d * NIJ);
            }
        }
#pragma unroll
        for (int d = 0; d < JK_MD_DENS; ++d) md_back<LK, LL>(Kx, Ky, Kz, jq[d], kq, jkl[d]);
    }
#pragma unroll
    for (int d = 0; d < JK_MD_DENS; ++d) {
        if (d >= n_j) break;
        double *jh = V.Jh + d * nao2;
#pragma unroll
        for (int c = 0; c < NK; ++c)
#pragma unroll
            for (int e = 0; e < NL; ++e)
                atomicAdd(jh + (kt.i0 + c) * nao + kt.j0 + e, fac * jkl[d][c * NL + e]);
    }
}
