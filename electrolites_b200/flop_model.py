"""Algorithmic flop count of a J/K build (the roofline numerator).

Per surviving shell quartet of class (li, lj | lk, ll) with n = (L/2) + 1
Rys roots, P = nprim_ij * nprim_kl primitive quartets,
g = nf_i nf_j nf_k nf_l Cartesian integrals:

    F_prim  = 30 + n (F_root + 3 F_2d + 3 g)
    F_root  = 2 * 13 * 2 = 52      (degree-13 Chebyshev, root and weight)
    F_2d    = 2 lij + 5 (lij+1) lkl + 2 (lkl+1) sum_{j=1..lj} (lij-j+1)
              + 2 (li+1)(lj+1) sum_{l=1..ll} (lkl-l+1)
    digest  = g * 2 * (4 n_k + 2 n_j)   (K: four contractions per density,
                                          J: two)
    total   = sum over quartets of P F_prim + digest

This is the count of the reference's per-primitive formulation (VRR, TRR
and HRR per root and primitive, 3 flops per integral per root), frozen so
that every form of the build is credited with the same work for the same
screened quartet list.  The engine's late transfer does fewer flops than
this for contracted shells, so the achieved rate it implies can exceed the
rate the hardware executes.
"""
from __future__ import annotations

F_PRIM_BASE = 30
F_ROOT = 52


def ncart(l):
    return (l + 1) * (l + 2) // 2


def f_2d(li, lj, lk, ll):
    lij, lkl = li + lj, lk + ll
    return (2 * lij + 5 * (lij + 1) * lkl
            + 2 * (lkl + 1) * sum(lij - j + 1 for j in range(1, lj + 1))
            + 2 * (li + 1) * (lj + 1) * sum(lkl - l + 1 for l in range(1, ll + 1)))


def nroots(li, lj, lk, ll):
    return (li + lj + lk + ll) // 2 + 1


def prim_flops(li, lj, lk, ll):
    g = ncart(li) * ncart(lj) * ncart(lk) * ncart(ll)
    return F_PRIM_BASE + nroots(li, lj, lk, ll) * (F_ROOT + 3 * f_2d(li, lj, lk, ll) + 3 * g)


def digest_flops(li, lj, lk, ll, n_j, n_k):
    g = ncart(li) * ncart(lj) * ncart(lk) * ncart(ll)
    return g * 2 * (4 * n_k + 2 * n_j)


def quartet_flops(li, lj, lk, ll, nprim_ij, nprim_kl, n_j, n_k):
    return (nprim_ij * nprim_kl * prim_flops(li, lj, lk, ll)
            + digest_flops(li, lj, lk, ll, n_j, n_k))


def build_flops(stats, n_j, n_k):
    """stats: {(li, lj, lk, ll): (quartets, primitive quartets)}."""
    total = 0
    for (li, lj, lk, ll), (nq, npq) in stats.items():
        total += npq * prim_flops(li, lj, lk, ll) + nq * digest_flops(li, lj, lk, ll, n_j, n_k)
    return total
