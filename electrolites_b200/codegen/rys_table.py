"""Rys quadrature roots and weights, and the Chebyshev tables the kernels read.

The two-electron integral over four Gaussians reduces to a one-dimensional
integral over t in [0, 1] with the weight exp(-x t^2).  Writing u = t^2, the
Rys nodes u_i and weights w_i of order n satisfy

    sum_i w_i u_i^m = F_m(x) = int_0^1 t^(2m) exp(-x t^2) dt,   m < 2n,

so sum_i w_i = F_0(x) (the Boys function) and the nodes live in (0, 1).  This
is the convention of the reference kernels (`rys_roots_reg`,
electrolites/kernels/fastk_prologue.cu:69-121): roots are t^2 and the weights
sum to F_0.

How the numbers here are made (no table is taken from anywhere else):

* `rys_exact(n, x)`: the measure is discretised with a composite
  Gauss-Legendre rule in t (panels graded towards t = 0 for large x), the
  three-term recurrence of the monic orthogonal polynomials in u is obtained by
  the discretised Stieltjes procedure, the nodes are the zeros of p_n (float64
  eigenvalues of the Jacobi matrix, polished by Newton steps on p_n in 80-bit
  long double) and the weights are the Christoffel numbers
  1 / sum_j p_j(u_i)^2 / ||p_j||^2.  All arithmetic is numpy longdouble.
* For x >= XMAX the interval [0, 1] may be replaced by [0, inf): the nodes
  become s_k^2 / x and the weights W_k / sqrt(x), with s_k the positive zeros
  of the Hermite polynomial H_2n and W_k their Gauss-Hermite weights.  XMAX is
  chosen so that the substitution changes no root or weight by more than
  1e-16 relative (checked by `check_asymptotic`).
* Below XMAX each of the 2n functions u_i(x), w_i(x) is fitted, per interval
  of width H, by a Chebyshev series of degree DEGREE interpolated at the
  Chebyshev points of that interval (order n: the intervals below its switch
  point XMAX_N[n-1] only).

Run as a script to write the C include file used by the CUDA build.
"""
from __future__ import annotations

import functools
import os
import sys

import numpy as np

LD = np.longdouble

NMAX = 7            # up to (ff|ff): floor(12/2) + 1 roots
# Interval layout of the piecewise Chebyshev fit: (start, end, width) per
# segment.  The roots vary fastest at small x, so the intervals are narrow
# there; degree 7 on these widths keeps every root and weight within ~2e-15
# relative for n <= 7 (8 coefficients: four 16-byte loads per row in the
# kernels, the data path being what the one-root classes wait on).
SEGMENTS = ((0.0, 10.0, 0.25), (10.0, 30.0, 0.5), (30.0, 100.0, 1.0))
XMAX = 100.0        # the segments cover [0, XMAX)
# Per order n, the argument from which the kernels switch to the Hermite
# limit: the substitution changes no root or weight by more than ~1e-16
# relative there (check_asymptotic; the fits themselves are ~1e-15), and
# every primitive quartet above it skips the table.  The table of order n
# holds the intervals below XMAX_N[n-1] only.
XMAX_N = (40.0, 50.0, 56.0, 62.0, 70.0, 78.0, 86.0)
NINT = sum(int(round((b - a) / h)) for a, b, h in SEGMENTS)
DEGREE = 7          # Chebyshev degree per interval (DEGREE + 1 coefficients)
DEGREE_F32 = 7      # degree of the single-precision table (mixed precision)


def nint(n: int) -> int:
    """Intervals the table of order n holds: those below XMAX_N[n-1]."""
    out = 0
    for a, b, h in SEGMENTS:
        if a >= XMAX_N[n - 1]:
            break
        out += int(round((min(b, XMAX_N[n - 1]) - a) / h))
    return out


# --------------------------------------------------------------------------
# Gauss-Legendre and Gauss-Hermite rules in long double
# --------------------------------------------------------------------------
@functools.lru_cache(maxsize=None)
def gauss_legendre_ld(m: int):
    """m-point Gauss-Legendre nodes/weights on [-1, 1] in long double."""
    x0, _ = np.polynomial.legendre.leggauss(m)
    x = x0.astype(LD)
    for _ in range(6):
        p0 = np.ones_like(x)
        p1 = x.copy()
        for k in range(2, m + 1):
            p0, p1 = p1, ((2 * k - 1) * x * p1 - (k - 1) * p0) / k
        dp = m * (x * p1 - p0) / (x * x - 1)
        x = x - p1 / dp
    p0 = np.ones_like(x)
    p1 = x.copy()
    for k in range(2, m + 1):
        p0, p1 = p1, ((2 * k - 1) * x * p1 - (k - 1) * p0) / k
    dp = m * (x * p1 - p0) / (x * x - 1)
    w = 2 / ((1 - x * x) * dp * dp)
    return x, w


@functools.lru_cache(maxsize=None)
def half_hermite_ld(n: int):
    """Positive zeros s_k of H_2n squared, and the matching Gauss-Hermite
    weights: int_0^inf exp(-s^2) f(s^2) ds = sum_k W_k f(s_k^2)."""
    s0, w0 = np.polynomial.hermite.hermgauss(2 * n)
    s = s0[s0 > 0].astype(LD)
    # Newton polish on the physicists' Hermite recurrence
    for _ in range(4):
        h0 = np.ones_like(s)
        h1 = 2 * s
        for k in range(1, 2 * n):
            h0, h1 = h1, 2 * s * h1 - 2 * k * h0
        dh = 2 * (2 * n) * h0
        s = s - h1 / dh
    h0 = np.ones_like(s)
    h1 = 2 * s
    for k in range(1, 2 * n):
        h0, h1 = h1, 2 * s * h1 - 2 * k * h0
    # W = 2^(N-1) N! sqrt(pi) / (N^2 H_{N-1}(s)^2) with N = 2n
    N = 2 * n
    fact = LD(1)
    for k in range(2, N + 1):
        fact *= k
    W = (LD(2) ** (N - 1)) * fact * np.sqrt(LD(np.pi)) / (N * N * h0 * h0)
    order = np.argsort(s)
    return (s * s)[order], W[order]


def _discrete_measure(x: float):
    """Nodes u_k = t_k^2 and weights of exp(-x t^2) dt on [0, 1]."""
    x = LD(x)
    # panels: uniform in t for small x, graded near t = 0 for large x
    width = min(LD(1), LD(8) / np.sqrt(max(x, LD(1))))
    edges = [LD(0)]
    while edges[-1] < 1:
        edges.append(min(LD(1), edges[-1] + width / 4))
    edges = np.array(edges, dtype=LD)
    gx, gw = gauss_legendre_ld(24)
    a, b = edges[:-1, None], edges[1:, None]
    t = (a + b) / 2 + (b - a) / 2 * gx[None, :]
    w = (b - a) / 2 * gw[None, :] * np.exp(-x * t * t)
    return (t * t).ravel(), w.ravel()


def _recurrence(u, w, n):
    """Monic recurrence alpha_j, beta_j (j < n) of a discrete measure."""
    alpha = np.zeros(n, dtype=LD)
    beta = np.zeros(n, dtype=LD)
    p_prev = np.zeros_like(u)
    p = np.ones_like(u)
    norm_prev = LD(1)
    for j in range(n):
        norm = np.sum(w * p * p)
        alpha[j] = np.sum(w * u * p * p) / norm
        beta[j] = norm if j == 0 else norm / norm_prev
        p_prev, p = p, (u - alpha[j]) * p - (beta[j] if j else 0) * p_prev
        norm_prev = norm
    return alpha, beta


def _nodes_weights(alpha, beta):
    n = len(alpha)
    J = np.diag(alpha.astype(np.float64))
    if n > 1:
        off = np.sqrt(beta[1:].astype(np.float64))
        J += np.diag(off, 1) + np.diag(off, -1)
    r = np.sort(np.linalg.eigvalsh(J)).astype(LD)
    for _ in range(4):
        p_prev = np.zeros_like(r)
        p = np.ones_like(r)
        dp_prev = np.zeros_like(r)
        dp = np.zeros_like(r)
        for j in range(n):
            b = beta[j] if j else LD(0)
            p_new = (r - alpha[j]) * p - b * p_prev
            dp_new = p + (r - alpha[j]) * dp - b * dp_prev
            p_prev, p = p, p_new
            dp_prev, dp = dp, dp_new
        r = r - p / dp
    # Christoffel numbers with the orthonormal polynomials
    s = np.zeros_like(r)
    p_prev = np.zeros_like(r)
    p = np.ones_like(r)
    nrm = beta[0]
    for j in range(n):
        s += p * p / nrm
        if j + 1 < n:
            b = beta[j] if j else LD(0)
            p_prev, p = p, (r - alpha[j]) * p - b * p_prev
            nrm = nrm * beta[j + 1]
    return r, 1 / s


def rys_exact(n: int, x: float):
    """(roots u_i = t_i^2, weights w_i), long double, ascending roots."""
    u, w = _discrete_measure(x)
    alpha, beta = _recurrence(u, w, n)
    return _nodes_weights(alpha, beta)


def rys_asymptotic(n: int, x: float):
    r, W = half_hermite_ld(n)
    x = LD(x)
    return r / x, W / np.sqrt(x)


def check_asymptotic(n: int, x: float = None) -> float:
    """Largest relative change of a root or weight of order n at x (default:
    the order's switch point XMAX_N) when [0, 1] is replaced by [0, inf)."""
    x = XMAX_N[n - 1] if x is None else x
    r0, w0 = rys_exact(n, x)
    r1, w1 = rys_asymptotic(n, x)
    return float(max(np.max(np.abs(r1 / r0 - 1)), np.max(np.abs(w1 / w0 - 1))))


# --------------------------------------------------------------------------
# Chebyshev fit
# --------------------------------------------------------------------------
def _cheb_coeffs(f_vals, deg):
    """Chebyshev interpolation coefficients from values at the deg+1
    Chebyshev points cos(pi (k + 1/2) / (deg + 1)), long double."""
    m = deg + 1
    k = np.arange(m, dtype=LD)
    theta = np.pi * (k + LD(0.5)) / m
    c = np.zeros(m, dtype=LD)
    for j in range(m):
        c[j] = 2 / LD(m) * np.sum(f_vals * np.cos(j * theta))
    c[0] /= 2
    return c


def intervals():
    """[(x_left, width)] of every interval, segment by segment."""
    out = []
    for a, b, h in SEGMENTS:
        n = int(round((b - a) / h))
        out += [(a + i * h, h) for i in range(n)]
    return out


def locate(x):
    """(interval index, local variable s in [-1, 1]) as the kernels compute
    them: segment by comparison, floor through the 1.5*2^52 rounding trick."""
    it0 = 0
    for a, b, h in SEGMENTS:
        if x < b:
            v = (x - a) / h
            k = int(np.floor(v))
            k = min(k, int(round((b - a) / h)) - 1)
            return it0 + k, 2.0 * (v - k) - 1.0
        it0 += int(round((b - a) / h))
    raise ValueError(x)


def fit_tables(deg: int = DEGREE, nmax: int = NMAX):
    """coef[n-1] has shape (NINT, 2n, deg+1): rows 0..n-1 are the roots,
    rows n..2n-1 the weights, on the intervals of SEGMENTS; the local
    variable of interval [a, a + h) is s = 2 (x - a)/h - 1."""
    m = deg + 1
    k = np.arange(m, dtype=LD)
    cheb_pts = np.cos(np.pi * (k + LD(0.5)) / m)
    out = []
    ivs = intervals()
    for n in range(1, nmax + 1):
        tab = np.zeros((nint(n), 2 * n, m), dtype=LD)
        for it, (a, h) in enumerate(ivs[:nint(n)]):
            xs = LD(a) + (cheb_pts + 1) * LD(h) / 2
            vals = np.array([np.concatenate(rys_exact(n, float(xv)))
                             for xv in xs])        # (m, 2n)
            for row in range(2 * n):
                tab[it, row] = _cheb_coeffs(vals[:, row], deg)
        out.append(tab)
    return out


def cheb_to_monomial(c):
    """sum_k c_k T_k(s) -> sum_k a_k s^k (long double)."""
    n = len(c)
    T = [np.zeros(n, dtype=LD) for _ in range(n)]
    T[0][0] = 1
    if n > 1:
        T[1][1] = 1
    for k in range(2, n):
        T[k][1:] += 2 * T[k - 1][:-1]
        T[k] -= T[k - 2]
    a = np.zeros(n, dtype=LD)
    for k in range(n):
        a += c[k] * T[k]
    return a


def monomial(tab):
    """Table of Chebyshev rows -> table of monomial rows, same shape."""
    out = np.empty_like(tab)
    for idx in np.ndindex(tab.shape[:-1]):
        out[idx] = cheb_to_monomial(tab[idx])
    return out


def estrin(a, s):
    """sum_k a_k s^k the way the kernels evaluate it (even degree count)."""
    a = np.asarray(a, dtype=np.float64)
    s = np.float64(s)
    p = [a[k] + a[k + 1] * s for k in range(0, len(a), 2)]
    s2 = s * s
    while len(p) > 1:
        q = [p[k] + (p[k + 1] * s2 if k + 1 < len(p) else 0.0) for k in range(0, len(p), 2)]
        p, s2 = q, s2 * s2
    return p[0]


def clenshaw(c, s):
    b1 = np.zeros_like(s)
    b2 = np.zeros_like(s)
    for cj in c[:0:-1]:
        b1, b2 = cj + 2 * s * b1 - b2, b1
    return c[0] + s * b1 - b2


def eval_table(tabs, n, x):
    """Evaluate the fitted table exactly as the kernels do (float64)."""
    x = float(x)
    if x >= XMAX_N[n - 1]:
        r, w = rys_asymptotic(n, x)
        return r.astype(np.float64), w.astype(np.float64)
    it, s = locate(x)
    c = tabs[n - 1][it].astype(np.float64)
    vals = np.array([clenshaw(c[row], np.float64(s)) for row in range(2 * n)])
    return vals[:n], vals[n:]


def fit_error(tabs, n, xs):
    worst = 0.0
    for x in xs:
        r0, w0 = rys_exact(n, x)
        r1, w1 = eval_table(tabs, n, x)
        e = max(np.max(np.abs(r1 / r0.astype(np.float64) - 1)),
                np.max(np.abs(w1 / w0.astype(np.float64) - 1)))
        worst = max(worst, float(e))
    return worst


# --------------------------------------------------------------------------
# C include writer
# --------------------------------------------------------------------------
def write_include(outdir: str) -> None:
    """Write rys_table_dims.inc (sizes, compile-time offsets) and
    rys_table_data.inc (the host copies of the tables) into outdir."""
    tabs = fit_tables(DEGREE)
    tabs32 = fit_tables(DEGREE_F32)
    offs, off = [], 0
    offs32, off32 = [], 0
    for n in range(1, NMAX + 1):
        offs.append(off)
        off += nint(n) * 2 * n * (DEGREE + 1)
        offs32.append(off32)
        off32 += nint(n) * 2 * n * (DEGREE_F32 + 1)
    dims = [
        '// Generated by electrolites_b200/codegen/rys_table.py -- do not edit.',
        '#pragma once',
        f'#define RYS_NMAX {NMAX}',
        f'#define RYS_XMAX {XMAX!r}',
        # segment boundaries, inverse widths and first interval of each
        f'#define RYS_SEG1 {SEGMENTS[1][0]!r}',
        f'#define RYS_SEG2 {SEGMENTS[2][0]!r}',
        f'#define RYS_IH0 {1.0 / SEGMENTS[0][2]!r}',
        f'#define RYS_IH1 {1.0 / SEGMENTS[1][2]!r}',
        f'#define RYS_IH2 {1.0 / SEGMENTS[2][2]!r}',
        f'#define RYS_IT1 {int(round((SEGMENTS[0][1] - SEGMENTS[0][0]) / SEGMENTS[0][2]))}',
        f'#define RYS_IT2 {int(round((SEGMENTS[0][1] - SEGMENTS[0][0]) / SEGMENTS[0][2])) + int(round((SEGMENTS[1][1] - SEGMENTS[1][0]) / SEGMENTS[1][2]))}',
        f'#define RYS_NINT {NINT}',
        f'#define RYS_DEGREE {DEGREE}',
        f'#define RYS_DEGREE_F32 {DEGREE_F32}',
        f'#define RYS_TABLE_SIZE {off}',
        f'#define RYS_TABLE32_SIZE {off32}',
        'template <int N> __host__ __device__ constexpr double rys_xmax()',
        '{ return ' + ' '.join(f'N == {n + 1} ? {x!r} :' for n, x in enumerate(XMAX_N)) + ' RYS_XMAX; }',
        'template <int N> __host__ __device__ constexpr int rys_nint()',
        '{ return ' + ' '.join(f'N == {n} ? {nint(n)} :' for n in range(1, NMAX + 1)) + ' -1; }',
        'template <int N> __host__ __device__ constexpr int rys_offset()',
        '{ return ' + ' '.join(f'N == {n + 1} ? {o} :' for n, o in enumerate(offs)) + ' -1; }',
        'template <int N> __host__ __device__ constexpr int rys32_offset()',
        '{ return ' + ' '.join(f'N == {n + 1} ? {o} :' for n, o in enumerate(offs32)) + ' -1; }',
    ]
    lines = ['// Generated by electrolites_b200/codegen/rys_table.py -- do not edit.',
             '// Piecewise Chebyshev fits of the Rys roots (t^2) and weights.',
             '#pragma once']
    # the kernels evaluate each row as a polynomial in s (Estrin's scheme),
    # so the Chebyshev series are converted to monomial coefficients here
    tabs = [monomial(t) for t in tabs]
    tabs32 = [monomial(t) for t in tabs32]
    flat = np.concatenate([t.astype(np.float64).ravel() for t in tabs])
    lines.append('static const double rys_table_host[RYS_TABLE_SIZE] = {')
    for i in range(0, len(flat), 4):
        lines.append('  ' + ', '.join(f'{v:.17e}' for v in flat[i:i + 4]) + ',')
    lines.append('};')
    flat32 = np.concatenate([t.astype(np.float32).ravel() for t in tabs32])
    lines.append('static const float rys_table32_host[RYS_TABLE32_SIZE] = {')
    for i in range(0, len(flat32), 6):
        lines.append('  ' + ', '.join(f'{v:.9e}f' for v in flat32[i:i + 6])
                     + ',')
    lines.append('};')
    r_rows, w_rows = [], []
    for n in range(1, NMAX + 1):
        r, W = half_hermite_ld(n)
        r_rows.append(list(r.astype(np.float64)) + [0.0] * (NMAX - n))
        w_rows.append(list(W.astype(np.float64)) + [0.0] * (NMAX - n))
    lines.append('static const double rys_largex_r_host[RYS_NMAX][RYS_NMAX] = {')
    for row in r_rows:
        lines.append('  {' + ', '.join(f'{v:.17e}' for v in row) + '},')
    lines.append('};')
    lines.append('static const double rys_largex_w_host[RYS_NMAX][RYS_NMAX] = {')
    for row in w_rows:
        lines.append('  {' + ', '.join(f'{v:.17e}' for v in row) + '},')
    lines.append('};')
    os.makedirs(outdir, exist_ok=True)
    for name, body in (('rys_table_dims.inc', dims), ('rys_table_data.inc', lines)):
        path = os.path.join(outdir, name)
        tmp = path + '.tmp'
        with open(tmp, 'w') as f:
            f.write('\n'.join(body) + '\n')
        os.replace(tmp, path)


if __name__ == '__main__':
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(
        os.path.dirname(os.path.abspath(__file__)), '..', 'csrc', 'generated')
    write_include(out)
