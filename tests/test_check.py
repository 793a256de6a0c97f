"""The fast FP64 checker (oracle/jk_check.c) against the long-double oracle.

The checker is what the GPU parity tests and bench.py compare the engine
with at the sizes the oracle cannot reach (a (H2O)_96 build is ~1.2e9
quartets), and the timed CPU baseline.  It restates the same arithmetic with
double-precision Rys roots (Chebyshev fits of the oracle's own long-double
solver) and a half-matrix digest; the oracle applies all eight index
permutations one by one.  Both must agree to 1e-12 on every J/K element
over all 55 classes, every hermi and J-only / K-only requests, and with the
committed (H2O)_8 fixture.
"""
import os

import numpy as np
import pytest

from electrolites_b200 import clusters
from electrolites_b200.gto import Mole

TOL = 1e-13
ATOL = 1e-12
GOLD = os.path.join(os.path.dirname(__file__), 'golden', 'h2o8_631gs_oracle.npz')


def all_class_mol():
    """Three centres carrying s, p, d and f shells of one and two
    primitives: every one of the 55 classes up to (ff|ff) occurs."""
    b = {
        'H': [[0, (1.3, 0.6), (0.3, 0.5)], [1, (0.9, 1.0)], [2, (0.7, 1.0)], [3, (0.6, 1.0)]],
        'He': [[0, (0.8, 1.0)], [1, (1.4, 0.7), (0.4, 0.4)], [2, (1.1, 1.0)], [3, (0.9, 1.0)]],
        'C': [[0, (2.1, 1.0)], [1, (0.5, 1.0)], [2, (0.9, 0.5), (0.35, 0.6)], [3, (1.2, 1.0)]],
    }
    atom = [('H', (0.0, 0.0, 0.0)), ('He', (0.9, 0.3, -0.4)), ('C', (-0.5, 1.1, 0.6))]
    return Mole(atom, basis=b, cart=True)


def _densities(mol, kind, rng):
    nao = mol.nao_cart
    D = clusters.atomic_density(mol, 1)
    if kind == 'uhf':
        return clusters.uhf_pair(D, 2)
    if kind == 'general':                       # hermi 0
        return np.stack([D + 0.01 * rng.standard_normal((nao, nao)), D])
    a = rng.standard_normal((nao, nao))         # hermi 2
    return (a - a.T)[None]


def test_checker_rys_roots_match_the_oracle_solver(oracle):
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.uniform(0, 100, 60), np.arange(0, 97, 4.0),
                         [1e-9, 95.999, 96.0, 96.001, 150.0, 1e3, 1e5]])
    for n in range(1, 8):
        for x in xs:
            r, w = oracle.rys(n, x)
            r2, w2 = oracle.check_rys(n, x)
            assert np.abs((r2 - r) / r).max() <= 1e-14, (n, x)
            assert np.abs((w2 - w) / w).max() <= 1e-14, (n, x)


@pytest.mark.parametrize('name,kind,combos', [
    ('spdf', 'uhf', 'all'), ('spdf', 'general', 'all'), ('spdf', 'antisymmetric', 'all'),
    ('h2o3', 'uhf', 'jk'), ('h2o3', 'general', 'jk'), ('h2o2_tzvp', 'uhf', 'jk')])
def test_checker_matches_oracle(oracle, name, kind, combos):
    mol = {'spdf': all_class_mol,
           'h2o3': lambda: clusters.water_mole(3, 5.0, 20261203, basis='6-31g*'),
           'h2o2_tzvp': lambda: clusters.water_mole(2, 4.0, 9, basis='def2-tzvp')}[name]()
    rng = np.random.default_rng(5)
    dms = _densities(mol, kind, rng)
    for wj, wk in ([(True, True), (True, False), (False, True)] if combos == 'all'
                   else [(True, True)]):
        rj, rk, nq = oracle.jk(mol, dms, tol=TOL, with_j=wj, with_k=wk)
        fj, fk, nq2 = oracle.jk_fast(mol, dms, tol=TOL, with_j=wj, with_k=wk)
        assert nq == nq2
        assert np.abs(fj - rj).max() <= ATOL
        assert np.abs(fk - rk).max() <= ATOL


def test_checker_matches_the_committed_fixture(oracle):
    g = np.load(GOLD)
    mol = clusters.water_mole(8, 7.0, int(g['seed']), basis='6-31g*', cart=True)
    fj, fk, nq = oracle.jk_fast(mol, g['dm'], tol=float(g['tol']))
    assert nq == int(g['nquartets'])
    assert np.abs(fj - g['vj']).max() <= ATOL
    assert np.abs(fk - g['vk']).max() <= ATOL


def test_checker_long_range_matches_oracle(oracle):
    mol = all_class_mol()
    dms = _densities(mol, 'uhf', None)
    rj, rk, _ = oracle.jk(mol, dms, tol=TOL, omega=0.4)
    fj, fk, _ = oracle.jk_fast(mol, dms, tol=TOL, omega=0.4)
    assert np.abs(fj - rj).max() <= ATOL
    assert np.abs(fk - rk).max() <= ATOL


def test_checker_integrals_match_oracle_per_quartet(oracle):
    """Single shell quartets in both shell orders (the checker stores each
    pair with its larger shell first and maps the block back)."""
    mol = all_class_mol()
    rng = np.random.default_rng(3)
    for _ in range(40):
        i, j, k, l = (int(v) for v in rng.integers(0, mol.nbas, 4))
        i, j = max(i, j), min(i, j)
        k, l = max(k, l), min(k, l)
        ref = oracle.eri_shells(mol, i, j, k, l)
        got = oracle.check_eri_shells(mol, i, j, k, l)
        assert np.abs(got - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max())


def test_checker_shards_sum_to_the_full_build(oracle):
    mol = clusters.water_mole(3, 5.0, 20261203, basis='6-31g*')
    dms = _densities(mol, 'uhf', None)
    fj, fk, nq = oracle.jk_fast(mol, dms, tol=TOL)
    sj, sk, snq = 0, 0, 0
    for s in range(3):
        a, b, n = oracle.jk_fast(mol, dms, tol=TOL, shard=s, nshard=3)
        sj, sk, snq = sj + a, sk + b, snq + n
    assert snq == nq
    assert np.abs(sj - fj).max() <= 1e-13 and np.abs(sk - fk).max() <= 1e-13


def _fd_gradient(oracle, mol, dms, jf, kf, atoms, h=2e-3):
    """Richardson-extrapolated central differences of the checker's energy
    E = j/2 Tr[Dt J[Dt]] - k c sum_s Tr[D_s K[D_s]] at displaced atoms."""
    g = np.zeros((len(atoms), 3))
    for ia, A in enumerate(atoms):
        ptr = mol._atm[A, 1]
        for x in range(3):
            e = {}
            for s in (-2, -1, 1, 2):
                mol._env[ptr + x] += s * h
                e[s] = oracle.jk_energy(mol, dms, jf, kf, tol=0)
                mol._env[ptr + x] -= s * h
            d1 = (e[1] - e[-1]) / (2 * h)
            d2 = (e[2] - e[-2]) / (4 * h)
            g[ia, x] = (4 * d1 - d2) / 3
    return g


@pytest.mark.parametrize('name', ['spdf', 'h2o2'])
def test_checker_gradient_matches_finite_differences(oracle, name):
    """The checker's nuclear gradient of the two-electron energy (derivative
    integrals from raised and lowered shells, up to g) against finite
    differences of its own J/K energies, RHF- and UHF-shaped, J and K terms
    apart; the forces sum to zero (translational invariance)."""
    mol = {'spdf': all_class_mol,
           'h2o2': lambda: clusters.water_mole(2, 4.0, 3, basis='6-31g*')}[name]()
    rng = np.random.default_rng(0)
    D = clusters.atomic_density(mol, 1) + 0.05 * rng.standard_normal((mol.nao_cart,) * 2)
    D = 0.5 * (D + D.T)
    for dms, jf, kf in [(D[None], 1.0, 0.2), (clusters.uhf_pair(D, 2), 1.0, 0.5),
                        (D[None], 0.0, 1.0)]:
        g, _ = oracle.grad_jk_fast(mol, dms, jf, kf, tol=0)
        fd = _fd_gradient(oracle, mol, dms, jf, kf, [0, 1])
        assert np.abs(g[:2] - fd).max() <= 1e-9 * max(1.0, np.abs(g).max())
        assert np.abs(g.sum(axis=0)).max() <= 1e-12
