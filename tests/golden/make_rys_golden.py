"""Write tests/golden/rys_reference_golden.npz from the reference's own table.

The reference evaluates Rys roots and weights from the packed table
electrolites/kernels/data/rys_roots_dat.npz with `rys_roots_reg<NROOTS>`
(electrolites/kernels/fastk_prologue.cu:69-121): a linear form for x < 3e-7,
the Hermite limit for x > 35 + 5n, the erf closed form for n = 1, and a
degree-13 Chebyshev series on intervals of width 2.5 otherwise.  This script
restates that evaluation in numpy, runs it on a fixed grid of x for
n = 1..7 and stores the result, so that the tests can pin this project's own
Rys roots (the oracle's and the kernels') to the reference's numbers without
the reference being present.

    python tests/golden/make_rys_golden.py /path/to/reference
"""
import math
import os
import sys

import numpy as np

if len(sys.argv) != 2:
    sys.exit('usage: python tests/golden/make_rys_golden.py /path/to/reference')
REF = sys.argv[1]
TABLE = os.path.join(REF, 'electrolites', 'kernels', 'data',
                     'rys_roots_dat.npz')
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)),
                   'rys_reference_golden.npz')

DEGREE, INTERVALS = 13, 40


def ref_rys(tab, n, x):
    """fastk_prologue.cu:69-121, restated (roots are t^2, weights sum F_0)."""
    off = n * (n - 1) // 2
    r, w = np.empty(n), np.empty(n)
    if x < 3e-7:
        for i in range(n):
            r[i] = tab['ROOT_SMALLX_R0'][off + i] + tab['ROOT_SMALLX_R1'][off + i] * x
            w[i] = tab['ROOT_SMALLX_W0'][off + i] + tab['ROOT_SMALLX_W1'][off + i] * x
        return r, w
    if x > 35 + n * 5:
        ix = 1 / math.sqrt(x)
        t = math.sqrt(math.pi / 4) * ix
        for i in range(n):
            r[i] = tab['ROOT_LARGEX_R_DATA'][off + i] * ix * ix
            w[i] = tab['ROOT_LARGEX_W_DATA'][off + i] * t
        return r, w
    if n == 1:
        ix = 1 / math.sqrt(x)
        f0 = math.sqrt(math.pi / 4) * ix * math.erf(x * ix)
        e = math.exp(-x)
        r[0] = .5 * ix * ix * (f0 - e) / f0
        w[0] = f0
        return r, w
    data = tab['ROOT_RW_DATA']
    base = (DEGREE + 1) * INTERVALS * (n * (n - 1))
    it = int(x * .4)
    u = (x - it * 2.5) * 0.8 - 1.
    u2 = u * 2.
    rw = np.empty(2 * n)
    for i in range(2 * n):
        c = data[base + i * (DEGREE + 1) * INTERVALS:]
        c0 = c[it + DEGREE * INTERVALS]
        c1 = c[it + (DEGREE - 1) * INTERVALS]
        for k in range(DEGREE - 2, 0, -2):
            c2 = c[it + k * INTERVALS] - c1
            c3 = c0 + c1 * u2
            c1 = c2 + c3 * u2
            c0 = c[it + (k - 1) * INTERVALS] - c3
        rw[i] = c0 + c1 * u
    return rw[0::2], rw[1::2]


def main():
    tab = dict(np.load(TABLE))
    rng = np.random.default_rng(20261203)
    xs = np.concatenate([
        [0.0, 1e-9, 2.9e-7, 3.1e-7, 1e-4, 0.01, 0.5, 1.0, 2.5, 5.0, 10.0,
         17.3, 33.3, 39.99, 40.01, 49.9, 50.1, 69.9, 70.1, 99.0, 120.0, 500.0],
        rng.uniform(0, 3, 40), rng.uniform(0, 100, 120)])
    out = {'x': xs}
    for n in range(1, 8):
        roots = np.empty((len(xs), n))
        weights = np.empty((len(xs), n))
        for k, x in enumerate(xs):
            roots[k], weights[k] = ref_rys(tab, n, float(x))
        out[f'roots{n}'] = roots
        out[f'weights{n}'] = weights
    np.savez_compressed(OUT, **out)
    print('wrote', OUT)


if __name__ == '__main__':
    main()
