"""Synthetic Gaussian basis sets with the shell structure of 6-31G*,
def2-SVP and def2-TZVP for H and O.

No basis-set library is available to this package, and the published
exponents and contraction coefficients are not reproduced here.  What the
J/K engine's cost and screening depend on is the *shape* of a basis: the
number of shells, their angular momenta, their primitive counts, and
exponents spread from tight core to diffuse valence.  Each named set below
keeps the shell structure of its namesake (angular momentum and primitive
count of every contracted shell, hence the AO and shell counts) and fills in
exponents as geometric sequences around a per-shell centre value, with
positive contraction weights from a fixed smooth profile.

Shell structures (l, primitives):
  6-31g*     H: s3 s1                  O: s6 s3 s1 p3 p1 d1
  def2-svp   H: s3 s1 p1               O: s5 s1 s1 p3 p1 d1
  def2-tzvp  H: s3 s1 s1 p1            O: s6 s2 s1 s1 s1 p4 p1 p1 d1 d1 f1

Per water that gives 10 / 14 / 19 shells and 19 / 25 / 48 Cartesian AOs
(18 / 24 / 43 spherical).
"""
from __future__ import annotations

import math

# (l, nprim, centre exponent, ratio between neighbouring exponents)
_SHAPES = {
    '6-31g*': {
        'H': [(0, 3, 1.3, 4.5), (0, 1, 0.16, 1)],
        'O': [(0, 6, 120.0, 4.2), (0, 3, 2.2, 3.2), (0, 1, 0.27, 1),
              (1, 3, 2.2, 3.2), (1, 1, 0.27, 1), (2, 1, 0.80, 1)],
    },
    'def2-svp': {
        'H': [(0, 3, 1.1, 4.5), (0, 1, 0.12, 1), (1, 1, 0.80, 1)],
        'O': [(0, 5, 150.0, 4.4), (0, 1, 0.95, 1), (0, 1, 0.30, 1),
              (1, 3, 3.5, 3.4), (1, 1, 0.27, 1), (2, 1, 1.20, 1)],
    },
    'def2-tzvp': {
        'H': [(0, 3, 3.0, 4.8), (0, 1, 0.33, 1), (0, 1, 0.10, 1),
              (1, 1, 0.80, 1)],
        'O': [(0, 6, 300.0, 4.6), (0, 2, 4.0, 3.0), (0, 1, 1.0, 1),
              (0, 1, 0.44, 1), (0, 1, 0.15, 1),
              (1, 4, 6.0, 3.6), (1, 1, 0.45, 1), (1, 1, 0.14, 1),
              (2, 1, 2.3, 1), (2, 1, 0.65, 1), (3, 1, 1.4, 1)],
    },
}
_ALIASES = {'6-31gs': '6-31g*', '631g*': '6-31g*', 'def2svp': 'def2-svp',
            'def2tzvp': 'def2-tzvp'}


def names():
    return sorted(_SHAPES)


def _key(name: str) -> str:
    k = name.lower().replace('_', '-')
    return _ALIASES.get(k, k)


def shells(name: str, element: str):
    """[[l, (exp, coef), ...], ...] for one element, PySCF's format."""
    table = _SHAPES[_key(name)]
    out = []
    for l, nprim, centre, ratio in table[element]:
        if nprim == 1:
            out.append([l, (centre, 1.0)])
            continue
        half = (nprim - 1) / 2
        prims = []
        for m in range(nprim):
            e = centre * ratio ** (half - m)
            # smooth positive weights peaking in the middle of the sequence
            w = math.exp(-0.35 * (m - half) ** 2) * (1 + 0.1 * m)
            prims.append((e, w))
        out.append([l] + prims)
    return out


def shell_structure(name: str, element: str):
    return [(l, n) for l, n, _, _ in _SHAPES[_key(name)][element]]
