"""Known-answer tests of the CPU oracle's integrals and J/K build.

The reference ships no golden J/K matrices (its tests compare live against
GPU4PySCF), so the oracle is pinned here by analytic results: the (ss|ss)
closed form through the Boys function, the Gaussian derivative identities
that turn s-type integrals into p- and d-type ones, the permutational
symmetry of (ij|kl) evaluated through different recurrence centres, and the
J/K conventions on small molecules."""
import math

import mpmath as mp
import numpy as np
import pytest

from electrolites_b200 import clusters
from electrolites_b200.gto import Mole, common_fac

SQRT_PI = math.sqrt(math.pi)


def boys0(t):
    if t < 1e-15:
        return 1.0
    return float(mp.sqrt(mp.pi / t) * mp.erf(mp.sqrt(t)) / 2)


def four_center_mol(exps, ls, coords):
    syms = ['H', 'He', 'C', 'N']
    basis = {s: [[l, (a, 1.0)]] for s, l, a in zip(syms, ls, exps)}
    atom = [(s, tuple(c)) for s, c in zip(syms, coords)]
    return Mole(atom, basis=basis, cart=True)


def raw_coef(mol, ish):
    b = mol._bas[ish]
    return mol._env[b[6]] * common_fac(int(b[1]))


def test_ssss_closed_form(oracle):
    rng = np.random.default_rng(3)
    for _ in range(5):
        exps = rng.uniform(0.1, 5, 4)
        coords = rng.uniform(-1.5, 1.5, (4, 3))
        mol = four_center_mol(exps, [0, 0, 0, 0], coords)
        R = mol.atom_coords()
        a, b, c, d = exps
        p, q = a + b, c + d
        P = (a * R[0] + b * R[1]) / p
        Q = (c * R[2] + d * R[3]) / q
        kab = math.exp(-a * b / p * np.sum((R[0] - R[1]) ** 2))
        kcd = math.exp(-c * d / q * np.sum((R[2] - R[3]) ** 2))
        T = p * q / (p + q) * np.sum((P - Q) ** 2)
        ref = 2 * math.pi ** 2.5 / (p * q * math.sqrt(p + q)) * kab * kcd * boys0(T)
        ref *= np.prod([raw_coef(mol, s) for s in range(4)])
        got = oracle.eri_shells(mol, 0, 1, 2, 3)[0, 0, 0, 0]
        assert abs(got - ref) <= 1e-14 * abs(ref)


def _raw_s(oracle, exps, coords):
    mol = four_center_mol(exps, [0, 0, 0, 0], coords)
    v = oracle.eri_shells(mol, 0, 1, 2, 3)[0, 0, 0, 0]
    return v / np.prod([raw_coef(mol, s) for s in range(4)])


def test_p_and_d_from_derivatives(oracle):
    """(x-Ax) e^{-a r_A^2} = (1/2a) d/dAx e^{-a r_A^2};
    (x-Ax)(y-Ay) e^{..} = (1/4a^2) d2/dAx dAy e^{..};
    (x-Ax)^2 e^{..} = (1/4a^2) (d2/dAx^2 + 2a) e^{..}  (coordinates in Bohr)."""
    rng = np.random.default_rng(11)
    exps = np.array([0.9, 1.3, 0.7, 1.1])
    coords = rng.uniform(-1, 1, (4, 3))       # Angstrom
    bohr = 1 / 0.52917721092
    h = 1e-3 / bohr                            # step in Angstrom, 1e-3 Bohr
    a = exps[0]

    def s_at(dx):
        c = coords.copy()
        c[0] += dx
        return _raw_s(oracle, exps, c)

    # p
    molp = four_center_mol(exps, [1, 0, 0, 0], coords)
    vp = oracle.eri_shells(molp, 0, 1, 2, 3)[:, 0, 0, 0]
    vp /= np.prod([raw_coef(molp, s) for s in range(4)])
    for d in range(3):
        e = np.zeros(3)
        e[d] = h
        fd1 = (s_at(e) - s_at(-e)) / (2 * h * bohr)
        fd2 = (s_at(e / 2) - s_at(-e / 2)) / (h * bohr)
        fd = (4 * fd2 - fd1) / 3            # Richardson: O(h^4)
        assert abs(vp[d] - fd / (2 * a)) <= 1e-8 * max(1e-3, abs(vp[d]))
    # d (xx, xy)
    mold = four_center_mol(exps, [2, 0, 0, 0], coords)
    vd = oracle.eri_shells(mold, 0, 1, 2, 3)[:, 0, 0, 0]
    vd /= np.prod([raw_coef(mold, s) for s in range(4)])
    ex, ey = np.array([h, 0, 0]), np.array([0, h, 0])
    s0 = s_at(np.zeros(3))
    d2xx = (s_at(ex) - 2 * s0 + s_at(-ex)) / (h * bohr) ** 2
    d2xy = (s_at(ex + ey) - s_at(ex - ey) - s_at(-ex + ey) + s_at(-ex - ey)) / (4 * (h * bohr) ** 2)
    assert abs(vd[0] - (d2xx + 2 * a * s0) / (4 * a * a)) <= 1e-5 * abs(vd[0])
    assert abs(vd[1] - d2xy / (4 * a * a)) <= 1e-5 * max(1e-3, abs(vd[1]))


@pytest.mark.parametrize('ls', [(1, 1, 1, 1), (2, 1, 2, 0), (3, 2, 1, 1), (3, 3, 2, 2),
                                (2, 2, 2, 2), (3, 0, 3, 1)])
def test_permutational_symmetry(oracle, ls):
    rng = np.random.default_rng(sum(ls))
    exps = rng.uniform(0.3, 2.0, 4)
    coords = rng.uniform(-1.2, 1.2, (4, 3))
    mol = four_center_mol(exps, list(ls), coords)
    v = oracle.eri_shells(mol, 0, 1, 2, 3)
    assert np.abs(v).max() > 0
    for perm, axes in [((1, 0, 2, 3), (1, 0, 2, 3)), ((0, 1, 3, 2), (0, 1, 3, 2)),
                       ((2, 3, 0, 1), (2, 3, 0, 1)), ((3, 2, 1, 0), (3, 2, 1, 0))]:
        w = oracle.eri_shells(mol, *perm)
        np.testing.assert_allclose(np.transpose(w, axes), v, rtol=1e-12,
                                   atol=1e-14 * np.abs(v).max())


def test_jk_conventions_small(oracle):
    """On one water: vj, vk symmetric for a symmetric density, E_J > 0,
    E_K < 0, screening changes nothing above 1e-12, and the general
    (non-symmetric) contraction follows dot_eri_dm's index convention."""
    mol = clusters.water_mole(1, 3.0, 5)
    D = clusters.atomic_density(mol, 1)
    vj, vk, nq = oracle.jk(mol, D, tol=0)
    assert np.allclose(vj, vj.T, atol=1e-13) and np.allclose(vk, vk.T, atol=1e-13)
    assert 0.5 * np.sum(D * vj) > 0 and -0.25 * np.sum(D * vk) < 0
    vj2, vk2, nq2 = oracle.jk(mol, D, tol=1e-13)
    assert nq2 <= nq
    assert np.abs(vj - vj2).max() < 1e-12 and np.abs(vk - vk2).max() < 1e-12
    # non-symmetric density: vk(D^T) = vk(D)^T, vj(D) = vj(sym(D))
    rng = np.random.default_rng(2)
    A = rng.standard_normal(D.shape) * 0.05
    vjA, vkA, _ = oracle.jk(mol, A, tol=0)
    vjT, vkT, _ = oracle.jk(mol, A.T.copy(), tol=0)
    np.testing.assert_allclose(vkT, vkA.T, atol=1e-13)
    np.testing.assert_allclose(vjT, vjA, atol=1e-13)


def test_jk_against_explicit_eri_tensor(oracle):
    """vj/vk from the oracle's J/K loop equal einsum over the full ERI tensor
    assembled shell by shell (two waters, 6-31G* shapes)."""
    mol = clusters.water_mole(2, 4.0, 9)
    nao = mol.nao_cart
    loc = mol.ao_loc_nr(cart=True)
    eri = np.zeros((nao,) * 4)
    nb = mol.nbas
    for i in range(nb):
        for j in range(nb):
            for k in range(nb):
                for l in range(nb):
                    eri[loc[i]:loc[i + 1], loc[j]:loc[j + 1], loc[k]:loc[k + 1],
                        loc[l]:loc[l + 1]] = oracle.eri_shells(mol, i, j, k, l)
    rng = np.random.default_rng(4)
    D = rng.standard_normal((nao, nao)) * 0.1
    vj, vk, _ = oracle.jk(mol, D, tol=0)
    np.testing.assert_allclose(vj, np.einsum('ijkl,ji->kl', eri, D), atol=1e-12)
    np.testing.assert_allclose(vk, np.einsum('ijkl,jk->il', eri, D), atol=1e-12)


def test_long_range_ssss_closed_form(oracle):
    """erf(omega r)/r: (ss|ss) = 2 pi^(5/2)/(p q sqrt(p+q)) K K' sqrt(theta)
    F_0(theta T), theta = omega^2/(omega^2 + rho) (the Boys function of the
    attenuated operator)."""
    rng = np.random.default_rng(5)
    for omega in (0.2, 0.9, 4.0):
        exps = rng.uniform(0.1, 5, 4)
        coords = rng.uniform(-1.5, 1.5, (4, 3))
        mol = four_center_mol(exps, [0, 0, 0, 0], coords)
        R = mol.atom_coords()
        a, b, c, d = exps
        p, q = a + b, c + d
        P = (a * R[0] + b * R[1]) / p
        Q = (c * R[2] + d * R[3]) / q
        kab = math.exp(-a * b / p * np.sum((R[0] - R[1]) ** 2))
        kcd = math.exp(-c * d / q * np.sum((R[2] - R[3]) ** 2))
        rho = p * q / (p + q)
        th = omega ** 2 / (omega ** 2 + rho)
        T = rho * np.sum((P - Q) ** 2)
        ref = 2 * math.pi ** 2.5 / (p * q * math.sqrt(p + q)) * kab * kcd * math.sqrt(th) * boys0(th * T)
        ref *= np.prod([raw_coef(mol, s) for s in range(4)])
        got = oracle.eri_shells(mol, 0, 1, 2, 3, omega=omega)[0, 0, 0, 0]
        assert abs(got - ref) <= 1e-14 * abs(ref)


@pytest.mark.parametrize('ls', [(1, 1, 1, 1), (3, 2, 2, 1), (3, 3, 3, 3)])
def test_long_range_limits(oracle, ls):
    """omega -> infinity gives the Coulomb integrals; the attenuated ones are
    permutation-symmetric like the Coulomb ones."""
    rng = np.random.default_rng(sum(ls) + 7)
    exps = rng.uniform(0.3, 2.0, 4)
    coords = rng.uniform(-1.2, 1.2, (4, 3))
    mol = four_center_mol(exps, list(ls), coords)
    full = oracle.eri_shells(mol, 0, 1, 2, 3)
    big = oracle.eri_shells(mol, 0, 1, 2, 3, omega=1e7)
    np.testing.assert_allclose(big, full, rtol=1e-9, atol=1e-12 * np.abs(full).max())
    lr = oracle.eri_shells(mol, 0, 1, 2, 3, omega=0.5)
    lr2 = np.transpose(oracle.eri_shells(mol, 2, 3, 0, 1, omega=0.5), (2, 3, 0, 1))
    np.testing.assert_allclose(lr2, lr, rtol=1e-12, atol=1e-14 * np.abs(lr).max())
    assert np.abs(lr).max() < np.abs(full).max()


def test_long_range_p_from_derivative(oracle):
    """(p s|s s) of the attenuated operator from the derivative of its s-type
    integral with respect to the first centre, as for 1/r."""
    rng = np.random.default_rng(13)
    exps = np.array([0.9, 1.3, 0.7, 1.1])
    coords = rng.uniform(-1, 1, (4, 3))
    bohr = 1 / 0.52917721092
    h = 1e-3 / bohr
    a, omega = exps[0], 0.6

    def s_at(dx):
        c = coords.copy()
        c[0] += dx
        mol = four_center_mol(exps, [0, 0, 0, 0], c)
        v = oracle.eri_shells(mol, 0, 1, 2, 3, omega=omega)[0, 0, 0, 0]
        return v / np.prod([raw_coef(mol, s) for s in range(4)])

    molp = four_center_mol(exps, [1, 0, 0, 0], coords)
    vp = oracle.eri_shells(molp, 0, 1, 2, 3, omega=omega)[:, 0, 0, 0]
    vp /= np.prod([raw_coef(molp, s) for s in range(4)])
    for d in range(3):
        e = np.zeros(3)
        e[d] = h
        fd1 = (s_at(e) - s_at(-e)) / (2 * h * bohr)
        fd2 = (s_at(e / 2) - s_at(-e / 2)) / (h * bohr)
        fd = (4 * fd2 - fd1) / 3
        assert abs(vp[d] - fd / (2 * a)) <= 1e-8 * max(1e-3, abs(vp[d]))
