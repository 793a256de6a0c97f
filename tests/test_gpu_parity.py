"""Parity of the CUDA J/K engine with the CPU oracle (through the C ABI).

Tolerances (plain FP64 form): every J/K element within 1e-10 absolute of
the oracle, and the J and K energies within 1e-9 Eh.  Shapes of the
reference's own tests (tests/test_jk.py:91-115 there): identical densities
must give identical results, random perturbations exercise the union
screening, atom-local densities the CPHF shape; hermi 1, 0 and 2; several
densities per call; an all-zero density must return zeros."""
import os

import numpy as np
import pytest

from electrolites_b200 import clusters
from electrolites_b200.gto import Mole

pytestmark = pytest.mark.gpu

ATOL = 1e-10
ETOL = 1e-9
TOL = 1e-13
GOLD = os.path.join(os.path.dirname(__file__), 'golden', 'h2o8_631gs_oracle.npz')


@pytest.fixture(scope='module')
def torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return torch


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


MOLS = {
    'h2o_631gs': lambda: clusters.water_mole(1, 3.0, 7, basis='6-31g*'),
    'h2o2_svp': lambda: clusters.water_mole(2, 4.5, 8, basis='def2-svp'),
    'h2o_tzvp': lambda: clusters.water_mole(1, 3.0, 9, basis='def2-tzvp'),
    'spdf': all_class_mol,
}


def densities(mol, kind, n_dm, hermi, rng):
    nao = mol.nao_cart
    base = clusters.atomic_density(mol, 11) if kind != 'atomic' else None
    out = np.empty((n_dm, nao, nao))
    for i in range(n_dm):
        if kind == 'same':
            out[i] = base
        elif kind == 'random':
            out[i] = base + 1e-2 * rng.standard_normal((nao, nao)) * 10. ** -(i % 3)
        else:
            out[i] = 0
            p0, p1 = mol.aoslice_by_atom(cart=True)[i % mol.natm][2:]
            out[i, p0:p1, p0:p1] = rng.standard_normal((p1 - p0, p1 - p0))
    if hermi == 1:
        out = out + out.transpose(0, 2, 1)
    elif hermi == 2:
        out = out - out.transpose(0, 2, 1)
    return out


def _energies(D, vj, vk):
    return 0.5 * np.einsum('nij,nji->', D, vj), -0.25 * np.einsum('nij,nji->', D, vk)


def _check(torch, opt, oracle, mol, dms, hermi, with_j=True, with_k=True):
    vj, vk = opt.get_jk(torch.as_tensor(dms), hermi, with_j=with_j, with_k=with_k)
    rj, rk, _ = oracle.jk(mol, dms, tol=TOL)
    if hermi == 2:
        rj = np.zeros_like(rj)
    if with_j:
        gj = vj.cpu().numpy()
        assert np.abs(gj - rj).max() <= ATOL, np.abs(gj - rj).max()
    if with_k:
        gk = vk.cpu().numpy()
        assert np.abs(gk - rk).max() <= ATOL, np.abs(gk - rk).max()
    if with_j and with_k:
        ej, ek = _energies(dms, gj, gk)
        rej, rek = _energies(dms, rj, rk)
        assert abs(ej - rej) <= ETOL and abs(ek - rek) <= ETOL
    return vj, vk


@pytest.mark.parametrize('name', list(MOLS))
@pytest.mark.parametrize('hermi', [1, 0, 2])
def test_parity_small(torch, oracle, name, hermi):
    from electrolites_b200.jk import VHFOpt
    mol = MOLS[name]()
    opt = VHFOpt(mol, TOL).build()
    rng = np.random.default_rng(20240908)
    for kind, n_dm in [('random', 1), ('random', 3), ('atomic', 2)]:
        dms = densities(mol, kind, n_dm, hermi, rng)
        _check(torch, opt, oracle, mol, dms, hermi)


@pytest.mark.parametrize('with_j,with_k', [(True, False), (False, True)])
def test_parity_j_only_k_only(torch, oracle, with_j, with_k):
    from electrolites_b200.jk import VHFOpt
    mol = MOLS['spdf']()
    opt = VHFOpt(mol, TOL).build()
    dms = densities(mol, 'random', 2, 1, np.random.default_rng(3))
    _check(torch, opt, oracle, mol, dms, 1, with_j, with_k)


def test_same_densities_identical(torch):
    """Identical densities come back identical (a wrong per-density stride
    cannot hide); differences are FP64 atomic-order round-off only."""
    from electrolites_b200.jk import VHFOpt
    mol = MOLS['h2o2_svp']()
    opt = VHFOpt(mol, TOL).build()
    dms = densities(mol, 'same', 4, 1, np.random.default_rng(0))
    vj, vk = opt.get_jk(torch.as_tensor(dms), 1)
    for v in (vj, vk):
        v = v.cpu().numpy()
        assert np.abs(v - v[0]).max() <= 1e-13 * np.abs(v).max()


def test_zero_density_returns_zeros(torch):
    from electrolites_b200.jk import VHFOpt
    mol = MOLS['h2o_631gs']()
    opt = VHFOpt(mol, TOL).build()
    z = torch.zeros((2, mol.nao_cart, mol.nao_cart), dtype=torch.float64)
    vj, vk = opt.get_jk(z, 1)
    assert float(vj.abs().max()) == 0.0 and float(vk.abs().max()) == 0.0


def test_schwarz_bounds(torch, oracle):
    from electrolites_b200.jk import VHFOpt
    mol = MOLS['spdf']()
    opt = VHFOpt(mol, TOL).build()
    q = opt.q_cond()
    ref = oracle.q_cond(mol)
    np.testing.assert_allclose(q, ref, rtol=0, atol=2e-6)


def test_cpu_workload_against_fixture(torch):
    """(H2O)_8 / 6-31G* shapes, atom-block density: the CPU-runnable
    workload, against the oracle's committed J/K."""
    from electrolites_b200.jk import VHFOpt
    g = np.load(GOLD)
    mol = clusters.water_mole(8, 7.0, int(g['seed']), basis='6-31g*')
    D = g['dm']
    opt = VHFOpt(mol, float(g['tol'])).build()
    vj, vk = opt.get_jk(torch.as_tensor(D), 1)
    vj, vk = vj.cpu().numpy(), vk.cpu().numpy()
    assert np.abs(vj - g['vj']).max() <= ATOL
    assert np.abs(vk - g['vk']).max() <= ATOL
    ej, ek = _energies(D[None], vj[None], vk[None])
    rej, rek = _energies(D[None], g['vj'][None], g['vk'][None])
    assert abs(ej - rej) <= ETOL and abs(ek - rek) <= ETOL
    nq = sum(v[0] for v in opt.class_counts().values())
    assert abs(nq - int(g['nquartets'])) <= 1e-3 * int(g['nquartets'])


def test_module_functions_spherical(torch, oracle):
    """get_jk(mol, dm) on a spherical-AO molecule: numpy in, numpy out,
    through the Cartesian transform."""
    from electrolites_b200 import jk
    mol = clusters.water_mole(1, 3.0, 4, basis='6-31g*', cart=False)
    C = mol.cart2sph_coeff()
    rng = np.random.default_rng(1)
    Ds = rng.standard_normal((mol.nao, mol.nao)) * 0.05
    Ds = Ds + Ds.T
    vj, vk = jk.get_jk(mol, Ds, hermi=1)
    assert isinstance(vj, np.ndarray) and vj.shape == Ds.shape
    rj, rk, _ = oracle.jk(mol, C @ Ds @ C.T, tol=TOL)
    np.testing.assert_allclose(vj, C.T @ rj @ C, atol=ATOL)
    np.testing.assert_allclose(vk, C.T @ rk @ C, atol=ATOL)
    np.testing.assert_allclose(jk.get_k(mol, Ds), vk, atol=1e-14)


def test_unsupported_requests_raise(torch):
    from electrolites_b200 import jk
    from electrolites_b200._lib import JKError
    mol = MOLS['h2o_631gs']()
    with pytest.raises(ValueError):   # mixing the ranges needs omega != 0
        jk.VHFOpt(mol).build().get_k(np.eye(mol.nao_cart), 1, omega=0.0, lr_factor=0.5,
                                     sr_factor=1.0)
    g = Mole([('H', (0, 0, 0))], basis={'H': [[4, (1.0, 1.0)]]}, cart=True)
    with pytest.raises(JKError, match='unsupported'):
        jk.VHFOpt(g).build()


def test_host_buffer_entry_point(torch, oracle):
    """jk_build_host: host density in, host J/K out."""
    import ctypes
    from electrolites_b200 import _lib
    from electrolites_b200.jk import VHFOpt
    mol = MOLS['h2o_tzvp']()
    opt = VHFOpt(mol, TOL).build()
    dms = densities(mol, 'random', 2, 1, np.random.default_rng(5))
    vj = np.zeros_like(dms)
    vk = np.zeros_like(dms)
    _lib.check(_lib.lib().jk_build_host(opt.plan, dms.ctypes.data, 2, 1, 1, 1,
                                        vj.ctypes.data, vk.ctypes.data, 0.0, None),
               'jk_build_host')
    rj, rk, _ = oracle.jk(mol, dms, tol=TOL)
    assert np.abs(vj - rj).max() <= ATOL and np.abs(vk - rk).max() <= ATOL


@pytest.mark.parametrize('name', ['h2o2_svp', 'spdf'])
def test_range_separated_operators(torch, oracle, name):
    """Long-range erf(omega r)/r (omega > 0), short-range erfc (omega < 0)
    and GPU4PySCF's lr/sr factor mixtures against the oracle (1e-10), on
    every class up to (ff|ff) for the s/p/d/f molecule."""
    from electrolites_b200.jk import VHFOpt
    mol = MOLS[name]()
    rng = np.random.default_rng(21)
    dms = densities(mol, 'random', 2, 1, rng)
    opt = VHFOpt(mol, TOL).build()
    w = 0.4
    fj, fk, _ = oracle.jk(mol, dms, tol=TOL)
    lj, lk, _ = oracle.jk(mol, dms, tol=TOL, omega=w)
    vj, vk = opt.get_jk(torch.as_tensor(dms), 1, omega=w)
    assert np.abs(vj.cpu().numpy() - lj).max() <= ATOL
    assert np.abs(vk.cpu().numpy() - lk).max() <= ATOL
    vj, vk = opt.get_jk(torch.as_tensor(dms), 1, omega=-w)
    assert np.abs(vj.cpu().numpy() - (fj - lj)).max() <= ATOL
    assert np.abs(vk.cpu().numpy() - (fk - lk)).max() <= ATOL
    vk = opt.get_k(torch.as_tensor(dms), 1, omega=w, lr_factor=0.8, sr_factor=0.2)
    ref = 0.8 * lk + 0.2 * (fk - lk)
    assert np.abs(vk.cpu().numpy() - ref).max() <= ATOL
    # the long-range operator is weaker: a smaller K energy in magnitude
    assert abs(np.einsum('nij,nji->', dms, lk)) < abs(np.einsum('nij,nji->', dms, fk))


@pytest.mark.parametrize('name', ['h2o2_svp', 'spdf'])
def test_fused_two_term_operator(torch, oracle, name):
    """One fused build of c0 op(0) + c1 op(w) (both terms inside the
    primitive loop, one screening and digest) equals the sum of the two
    one-term builds (1e-12) and the oracle's (1e-10), for J and K of a
    general (hermi 0) density; FP32 quartets of the mixed form keep the
    energies within 1e-7 Eh."""
    from electrolites_b200.jk import VHFOpt
    mol = MOLS[name]()
    dms = densities(mol, 'random', 2, 0, np.random.default_rng(23))
    opt = VHFOpt(mol, TOL).build()
    d = torch.as_tensor(dms, device='cuda')
    c0, c1, w = 0.35, -1.25, 0.3
    fj, fk = opt.build_jk_async(d, 0, terms=[(c0, 0.0), (c1, w)])
    aj, ak = opt.build_jk_async(d, 0, terms=[(c0, 0.0)])
    bj, bk = opt.build_jk_async(d, 0, terms=[(c1, w)])
    opt.sync()
    assert float((fj - aj - bj).abs().max()) <= 1e-12
    assert float((fk - ak - bk).abs().max()) <= 1e-12
    rj, rk, _ = oracle.jk(mol, dms, tol=TOL)
    lj, lk, _ = oracle.jk(mol, dms, tol=TOL, omega=w)
    assert np.abs(fj.cpu().numpy() - (c0 * rj + c1 * lj)).max() <= ATOL
    assert np.abs(fk.cpu().numpy() - (c0 * rk + c1 * lk)).max() <= ATOL
    mj, mk = opt.build_jk_async(d, 0, mixed_threshold=1e-6, terms=[(c0, 0.0), (c1, w)])
    opt.sync()
    ej, ek = _energies(dms, fj.cpu().numpy(), fk.cpu().numpy())
    mej, mek = _energies(dms, mj.cpu().numpy(), mk.cpu().numpy())
    assert abs(ej - mej) <= 1e-7 and abs(ek - mek) <= 1e-7


def test_operator_arguments_rejected(torch):
    from electrolites_b200 import _lib
    from electrolites_b200.jk import VHFOpt
    mol = MOLS['h2o2_svp']()
    opt = VHFOpt(mol, TOL).build()
    d = torch.zeros((1, mol.nao_cart, mol.nao_cart), dtype=torch.float64, device='cuda')
    with pytest.raises(ValueError):
        opt.build_jk_async(d, 1, terms=[(1.0, 0.0), (1.0, 0.2), (1.0, 0.3)])
    with pytest.raises(_lib.JKError, match='omega'):
        opt.build_jk_async(d, 1, terms=[(1.0, 0.0), (1.0, -0.2)])
    with pytest.raises(_lib.JKError, match='coefficients'):
        opt.build_jk_async(d, 1, terms=[(float('nan'), 0.0)])
    vj, vk = opt.get_jk(d, 1)
    assert float(vk.abs().max()) == 0.0


@pytest.mark.parametrize('name', ['spdf', 'h2o_tzvp'])
def test_j_engine(torch, oracle, name):
    """J-only builds through the J engine (the quartets' (e0|f0) blocks
    contracted with the pairs' x-space densities, transfers once per pair)
    against the oracle's J-only build (1e-10) and the (ij|kl) digest
    (1e-12), for symmetric and general densities, three of them; every class
    up to (ff|ff) (register and team forms) for the s/p/d/f molecule.  Mixed
    precision keeps E_J within 1e-7 Eh."""
    from electrolites_b200.jk import VHFOpt
    mol = MOLS[name]()
    opt = VHFOpt(mol, TOL).build()
    rng = np.random.default_rng(41)
    for hermi in (1, 0):
        dms = densities(mol, 'random', 3, hermi, rng)
        d = torch.as_tensor(dms, device='cuda')
        vj, vk = opt.get_jk(d, hermi, with_k=False)
        assert vk is None
        rj, _, _ = oracle.jk(mol, dms, tol=TOL, with_k=False)
        assert np.abs(vj.cpu().numpy() - rj).max() <= ATOL
        opt.set_jengine(False)
        dj, _ = opt.get_jk(d, hermi, with_k=False)
        opt.set_jengine(True)
        assert float((vj - dj).abs().max()) <= 1e-12
    mj, _ = opt.get_jk(d, 0, with_k=False, mixed_threshold=1e-6)
    ej = 0.5 * float((d * vj).sum())
    assert abs(0.5 * float((d * mj).sum()) - ej) <= 1e-7


class _GeneralContraction:
    """A molecule in PySCF's layout whose shells carry several contractions
    (nctr > 1): built from a molecule with one contraction per shell by
    merging runs of shells on one atom with the same l and exponents.  The
    AO order (contraction-major inside a shell) equals the split one."""

    def __init__(self, split):
        bas, env = [], list(split._env)
        rows = [list(r) for r in split._bas]
        s = 0
        while s < len(rows):
            ia, l, nprim, _, _, pe, pc, _ = rows[s]
            e = s + 1
            while (e < len(rows) and rows[e][0] == ia and rows[e][1] == l
                   and rows[e][2] == nprim
                   and list(split._env[rows[e][5]:rows[e][5] + nprim]) ==
                   list(split._env[pe:pe + nprim])):
                e += 1
            pc_new = len(env)
            for t in range(s, e):
                env.extend(split._env[rows[t][6]:rows[t][6] + nprim])
            bas.append([ia, l, nprim, e - s, 0, pe, pc_new, 0])
            s = e
        self._atm = split._atm
        self._bas = np.asarray(bas, dtype=np.int32)
        self._env = np.asarray(env)
        self.nbas = len(bas)
        self.cart = True

    def ao_loc_nr(self, cart=True):
        n = [(l + 1) * (l + 2) // 2 * nctr for l, nctr in zip(self._bas[:, 1], self._bas[:, 3])]
        return np.concatenate([[0], np.cumsum(n)]).astype(np.int32)


def test_general_contractions(torch, oracle):
    """Shells with several contractions are expanded contraction-major, as
    PySCF orders their AOs: J/K equal the oracle on the split molecule."""
    from electrolites_b200.jk import VHFOpt
    b = {'C': [[1, (1.2, 0.5), (0.4, 0.4), (0.1, 0.2)],
               [1, (1.2, -0.3), (0.4, 0.2), (0.1, 0.7)],
               [0, (3.0, 0.6), (0.7, 0.5)],
               [0, (3.0, 0.1), (0.7, -0.9)],
               [2, (0.8, 1.0)]],
         'H': [[0, (1.3, 0.6), (0.3, 0.5)], [1, (0.9, 1.0)]]}
    split = Mole([('C', (0.0, 0.0, 0.0)), ('H', (0.7, 0.5, -0.4)), ('H', (-0.8, 0.3, 0.6))],
                 basis=b, cart=True)
    gc = _GeneralContraction(split)
    assert gc.nbas < split.nbas and int(gc._bas[:, 3].max()) == 2
    rng = np.random.default_rng(31)
    dms = densities(split, 'random', 2, 0, rng)
    rj, rk, _ = oracle.jk(split, dms, tol=TOL)
    vj, vk = VHFOpt(gc, TOL).build().get_jk(torch.as_tensor(dms), 0)
    assert np.abs(vj.cpu().numpy() - rj).max() <= ATOL
    assert np.abs(vk.cpu().numpy() - rk).max() <= ATOL


# ---------------------------------------------------------------------------
# Parity at the sizes the benchmark times, against the fast FP64 checker
# (oracle/jk_check.c, itself checked against the long-double oracle to 1e-12
# in tests/test_check.py)
# ---------------------------------------------------------------------------
BENCH_SHAPES = {
    # (waters, cube edge A, basis, UHF pair, seed): the bench's workloads
    'h2o32_631gs_uhf': (32, 10.4, '6-31g*', True, 20261204),
    'h2o8_tzvp': (8, 6.5, 'def2-tzvp', False, 20261205),
    'h2o96_631gs_uhf': (96, 15.0, '6-31g*', True, 20261204),
}


def _bench_inputs(name):
    n, edge, basis, uhf, seed = BENCH_SHAPES[name]
    mol = clusters.water_mole(n, edge, seed, basis=basis, cart=True)
    D = clusters.atomic_density(mol, seed)
    dms = clusters.uhf_pair(D, seed + 1) if uhf else D[None]
    return mol, np.ascontiguousarray(dms)


@pytest.mark.parametrize('name', list(BENCH_SHAPES))
def test_parity_at_bench_sizes(torch, oracle, name):
    """Plain FP64 J/K of the benchmark's shapes -- (H2O)_32 6-31G* UHF,
    (H2O)_8 def2-TZVP, and the headline (H2O)_96 6-31G* UHF build itself --
    within 1e-10 of the checker on every element and 1e-9 Eh on E_J, E_K."""
    from electrolites_b200.jk import VHFOpt
    mol, dms = _bench_inputs(name)
    opt = VHFOpt(mol, TOL).build()
    vj, vk = opt.get_jk(torch.as_tensor(dms, device='cuda'), 1)
    gj, gk = vj.cpu().numpy(), vk.cpu().numpy()
    rj, rk, _ = oracle.jk_fast(mol, dms, tol=TOL)
    assert np.abs(gj - rj).max() <= ATOL, np.abs(gj - rj).max()
    assert np.abs(gk - rk).max() <= ATOL, np.abs(gk - rk).max()
    ej, ek = _energies(dms, gj, gk)
    rej, rek = _energies(dms, rj, rk)
    assert abs(ej - rej) <= ETOL and abs(ek - rek) <= ETOL, (ej - rej, ek - rek)


@pytest.mark.parametrize('seed', [34, 35])
def test_mixed_form_team_classes(torch, oracle, seed):
    """FP32 quartets of the mixed form in the team-form classes (the f-shell
    and (dd|ds)-and-larger classes), on a spread-out (H2O)_4 def2-TZVP
    cluster whose distant quartets fall below the threshold: at 1e-6 some
    team-class quartets run in FP32 and the J/K energies stay within 1e-7 Eh
    of the checker's; with the threshold off no quartet runs in FP32."""
    import ctypes

    from electrolites_b200 import _lib
    from electrolites_b200.jk import VHFOpt, class_keys
    mol = clusters.water_mole(4, 8.0, seed, basis='def2-tzvp')
    dms = clusters.uhf_pair(clusters.atomic_density(mol, seed), seed + 1)
    opt = VHFOpt(mol, TOL).build()
    d = torch.as_tensor(dms, device='cuda')
    forms = {}
    for k in range(len(class_keys())):
        ls = [ctypes.c_int() for _ in range(5)]
        _lib.lib().jk_class_info(k, *[ctypes.byref(x) for x in ls])
        forms[tuple(x.value for x in ls[:4])] = ls[4].value
    mj, mk = opt.get_jk(d, 1, mixed_threshold=1e-6)
    counts = opt.class_counts(with_f32=True)
    assert sum(c[2] for k, c in counts.items() if forms[k] == 1) > 0
    rj, rk, _ = oracle.jk_fast(mol, dms, tol=TOL)
    ej, ek = _energies(dms, rj, rk)
    mej, mek = _energies(dms, mj.cpu().numpy(), mk.cpu().numpy())
    assert abs(ej - mej) <= 1e-7 and abs(ek - mek) <= 1e-7
    opt.get_jk(d, 1)
    assert sum(c[2] for c in opt.class_counts(with_f32=True).values()) == 0
