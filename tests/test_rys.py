"""Rys roots and weights: the oracle's and the kernels' tables against the
reference's own table (golden vectors) and against Boys-function moments."""
import os

import mpmath as mp
import numpy as np
import pytest

from electrolites_b200.codegen import rys_table as R

GOLDEN = os.path.join(os.path.dirname(__file__), 'golden', 'rys_reference_golden.npz')


def boys(m, x):
    x = mp.mpf(x)
    if x == 0:
        return mp.mpf(1) / (2 * m + 1)
    return mp.gammainc(m + mp.mpf(0.5), 0, x) / (2 * x ** (m + mp.mpf(0.5)))


@pytest.mark.parametrize('n', [1, 2, 4, 7])
@pytest.mark.parametrize('x', [0.0, 1e-9, 0.37, 3.0, 18.0, 61.0, 99.5, 140.0])
def test_exact_roots_reproduce_boys_moments(n, x):
    mp.mp.dps = 30
    r, w = R.rys_exact(n, x)
    for m in range(2 * n):
        got = mp.mpf(float(np.sum(w * r ** m)))
        ref = boys(m, x)
        assert abs(got - ref) / ref < 5e-16


def test_oracle_roots_match_reference_golden(oracle):
    """The reference's table (electrolites/kernels/data/rys_roots_dat.npz,
    evaluated as electrolites/kernels/fastk_prologue.cu:69-121 does) agrees
    with the oracle's roots to its own accuracy: ~1e-11 relative, and ~1e-9
    for n = 1 just above its small-x switch, where its closed form cancels."""
    g = np.load(GOLDEN)
    for n in range(1, 8):
        tol = 2e-9 if n == 1 else 2e-11
        for k, x in enumerate(g['x']):
            r, w = oracle.rys(n, float(x))
            rr, ww = g[f'roots{n}'][k], g[f'weights{n}'][k]
            o = np.argsort(rr)
            np.testing.assert_allclose(r, rr[o], rtol=tol, atol=0)
            np.testing.assert_allclose(w, ww[o], rtol=tol, atol=0)


def test_table_fit_accuracy():
    """The kernels' piecewise Chebyshev table reproduces the exact roots to
    ~1e-15 relative over [0, XMAX) and uses the exact Hermite limit above."""
    tabs = R.fit_tables(R.DEGREE, nmax=3)
    rng = np.random.default_rng(7)
    xs = np.concatenate([rng.uniform(0, R.XMAX, 60), [0.0, 1e-10, R.XMAX - 1e-9],
                         [v - 1e-9 for v in R.XMAX_N[:3]], list(R.XMAX_N[:3])])
    for n in range(1, 4):
        assert R.fit_error(tabs, n, xs) < 5e-15
    for n in range(1, 8):
        assert R.check_asymptotic(n, R.XMAX) < 1e-15
        # the kernels switch to the Hermite limit at XMAX_N[n-1] <= XMAX
        assert R.XMAX_N[n - 1] <= R.XMAX
        for x in (R.XMAX_N[n - 1], R.XMAX_N[n - 1] + 3.0):
            assert R.check_asymptotic(n, x) < 5e-16


def test_table_include_matches_fit(tmp_path):
    """The generated include holds the fitted numbers (spot check)."""
    R.write_include(str(tmp_path))
    dims = (tmp_path / 'rys_table_dims.inc').read_text()
    assert f'#define RYS_DEGREE {R.DEGREE}' in dims
    data = (tmp_path / 'rys_table_data.inc').read_text()
    assert 'rys_table_host' in data and 'rys_largex_w_host' in data
