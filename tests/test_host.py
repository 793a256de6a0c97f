"""Host-side logic: basis shapes and normalisation, cluster geometry,
densities, the Cartesian->spherical transform, the C-ABI library exports,
the patch registry, and the flop model."""
import ctypes
import os
import re
import sys
import types

import numpy as np
import pytest

from electrolites_b200 import basis_synth, clusters, gto

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize('basis,nsh,ncart,nsph', [('6-31g*', 10, 19, 18),
                                                  ('def2-svp', 12, 25, 24),
                                                  ('def2-tzvp', 19, 48, 43)])
def test_basis_shapes(basis, nsh, ncart, nsph):
    mol = clusters.water_mole(1, 3.0, 1, basis=basis)
    assert mol.nbas == nsh
    assert mol.nao_cart == ncart
    assert mol.ao_loc_nr(cart=False)[-1] == nsph


def test_normalisation():
    mol = clusters.water_mole(1, 3.0, 2, basis='def2-tzvp')
    S = mol.intor_ovlp_cart()
    loc = mol.ao_loc_nr(True)
    for ish, l in enumerate(mol._bas[:, 1]):
        if l < 2:   # s and p Cartesian functions are normalised
            d = np.diag(S)[loc[ish]:loc[ish + 1]]
            np.testing.assert_allclose(d, 1.0, rtol=1e-12)
    C = mol.cart2sph_coeff()
    Ssph = C.T @ S @ C
    np.testing.assert_allclose(np.diag(Ssph), 1.0, rtol=1e-10)


def test_cluster_geometry():
    atoms = clusters.water_cluster(24, 3.1 * 24 ** (1 / 3), 42)
    O = np.array([xyz for s, xyz in atoms if s == 'O'])
    d = np.linalg.norm(O[:, None] - O[None], axis=-1) + np.eye(len(O)) * 99
    assert d.min() >= 2.7
    H = np.array([xyz for s, xyz in atoms if s == 'H']).reshape(-1, 2, 3)
    np.testing.assert_allclose(np.linalg.norm(H - O[:, None], axis=-1), 0.9572, rtol=1e-12)
    v1, v2 = H[:, 0] - O, H[:, 1] - O
    ang = np.degrees(np.arccos(np.sum(v1 * v2, 1) / 0.9572 ** 2))
    np.testing.assert_allclose(ang, 104.52, rtol=1e-10)
    assert clusters.water_cluster(24, 3.1 * 24 ** (1 / 3), 42) == atoms   # seeded


def test_density_electron_count():
    mol = clusters.water_mole(3, 5.0, 3)
    D = clusters.atomic_density(mol, 3)
    S = mol.intor_ovlp_cart()
    assert abs(np.trace(D @ S) - 30) < 1e-10
    np.testing.assert_allclose(D, D.T, atol=1e-14)
    da, db = clusters.uhf_pair(D, 5)
    np.testing.assert_allclose(da, 0.5 * D)
    np.testing.assert_allclose(db, db.T, atol=1e-15)
    assert 0 < np.abs(db - da).max() < 0.02 * np.abs(da).max()


def _header_symbols():
    text = open(os.path.join(ROOT, 'include', 'jk_b200.h')).read()
    return sorted(set(re.findall(r'^\s*(?:int|const char \*)\s*(jk_\w+)\s*\(', text, re.M)))


def test_library_exports_every_header_symbol():
    from electrolites_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip('library not built')
    L = ctypes.CDLL(_lib.LIB_PATH)
    syms = _header_symbols()
    assert 'jk_build' in syms and 'jk_plan_create' in syms
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) <= set(_lib.EXPORTS)


def test_library_errors_without_device_or_bad_args():
    """Argument errors come back as codes with a message; no silent path."""
    from electrolites_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip('library not built')
    L = _lib.lib()
    plan = ctypes.c_void_p()
    rc = L.jk_plan_create(None, 0, None, 0, None, None, 1e-13, 0, ctypes.byref(plan))
    assert rc != 0 and plan.value is None
    assert len(L.jk_last_error()) > 0
    assert L.jk_build(None, None, 1, 1, 1, 1, None, None, 0.0, None) == 1


def test_package_fails_loudly_without_library(monkeypatch):
    from electrolites_b200 import _lib
    monkeypatch.setattr(_lib, 'LIB_PATH', '/nonexistent/libjk_b200.so')
    monkeypatch.setattr(_lib, '_lib', None)
    with pytest.raises(RuntimeError, match='not built'):
        _lib.lib()


def test_patch_registry(monkeypatch):
    import electrolites_b200 as eb
    status = eb.check_targets()
    assert set(status) == set(eb.MODULES)
    if any(v is not None for v in status.values()):
        with pytest.raises(ImportError):
            eb.patch('fastjk')
    # a stand-in for gpu4pyscf's option classes
    pkg = types.ModuleType('gpu4pyscf')
    scf = types.ModuleType('gpu4pyscf.scf')
    jkm = types.ModuleType('gpu4pyscf.scf.jk')
    jem = types.ModuleType('gpu4pyscf.scf.j_engine')

    class Opt:
        def get_jk(self, dms, hermi, verbose=None):
            return 'orig'

        def get_k(self, dms, hermi, verbose=None, omega=None, lr_factor=None, sr_factor=None):
            return 'orig'

    class OptJ:
        def get_j(self, dms, verbose=None):
            return 'orig'

    jkm._VHFOpt, jem._VHFOpt = Opt, OptJ
    grad = types.ModuleType('gpu4pyscf.grad')
    grm = types.ModuleType('gpu4pyscf.grad.rhf')
    grm._jk_energy_per_atom = lambda vhfopt, dm, j_factor=1., k_factor=1., verbose=None: 'orig'
    for name, m in [('gpu4pyscf', pkg), ('gpu4pyscf.scf', scf), ('gpu4pyscf.scf.jk', jkm),
                    ('gpu4pyscf.scf.j_engine', jem), ('gpu4pyscf.grad', grad),
                    ('gpu4pyscf.grad.rhf', grm)]:
        monkeypatch.setitem(sys.modules, name, m)
    monkeypatch.setattr(eb, '_PATCHED', {})
    assert all(v is None for v in eb.check_targets().values())
    with pytest.raises(KeyError):
        eb.patch('nope')
    eb.patch_all()
    assert eb.patched() == sorted(eb.MODULES)
    assert Opt.get_jk is eb._get_jk and OptJ.get_j is eb._get_j
    assert grm._jk_energy_per_atom is eb._jk_energy_per_atom


def test_flop_model_counts():
    from electrolites_b200 import flop_model as F
    # (ss|ss), 1x1 primitives, 1 density, J+K
    f = F.quartet_flops(0, 0, 0, 0, 1, 1, n_j=1, n_k=1)
    assert f == F.F_PRIM_BASE + 1 * (F.F_ROOT + 3 * F.f_2d(0, 0, 0, 0) + 3 * 1) + 1 * 1 * 2 * 6
    assert F.quartet_flops(2, 2, 2, 2, 1, 1, 1, 1) > F.quartet_flops(1, 1, 1, 1, 1, 1, 1, 1)


def test_patched_methods_take_omega_from_the_option_mol(monkeypatch):
    """After patching, a range-separated functional's omega set on the option
    object's mol reaches the engine when the call names none (the reference
    resolves it there, electrolites/compat.py:178-187); an explicit omega
    wins."""
    import electrolites_b200 as eb
    seen = []

    class Plan:
        def get_jk(self, dms, hermi, verbose=None, omega=None):
            seen.append(('jk', omega))
            return dms, dms

        def get_k(self, dms, hermi, verbose=None, omega=None, lr_factor=None, sr_factor=None):
            seen.append(('k', omega, lr_factor, sr_factor))
            return dms

    class Opt:
        pass

    opt = Opt()
    opt.mol = types.SimpleNamespace(omega=0.3)
    opt._jk_b200 = Plan()
    eb._get_jk(opt, 'D', 1)
    eb._get_k(opt, 'D', 1)
    eb._get_k(opt, 'D', 1, None, -0.2, 1.0, 0.25)
    opt.mol = types.SimpleNamespace(omega=0.0)
    eb._get_k(opt, 'D', 1)
    assert seen == [('jk', 0.3), ('k', 0.3, None, None), ('k', -0.2, 1.0, 0.25),
                    ('k', None, None, None)]
    # the long-range operator of omega = 0.3 is one erf term
    from electrolites_b200.jk import _rsh_terms
    assert _rsh_terms(0.3, None, None) == [(1.0, 0.3)]


def test_module_plan_cache_follows_the_geometry():
    """The module functions' plan cache is keyed by the molecule's content:
    moving an atom in place changes the key, an unchanged molecule keeps it."""
    from electrolites_b200 import clusters
    from electrolites_b200.jk import _opt_key
    mol = clusters.water_mole(2, 4.0, 3, basis='6-31g*')
    k0 = _opt_key(mol)
    assert _opt_key(mol) == k0
    ptr = mol._atm[0, 1]
    mol._env[ptr] += 0.1
    assert _opt_key(mol) != k0
    mol._env[ptr] -= 0.1
    assert _opt_key(mol) == k0


def test_patched_gradient_target(monkeypatch):
    """The patched grad.rhf._jk_energy_per_atom brings the density to the
    option's sorted Cartesian basis through the option object and takes the
    operator's omega from the option's molecule (the reference's fastejk,
    electrolites/fastejk.py:270-276)."""
    import numpy as np

    import electrolites_b200 as eb
    seen = []

    class G:
        def cpu(self):
            return self

        def numpy(self):
            return np.zeros((2, 3))

    class Plan:
        def jk_energy_per_atom(self, dms, j, k, omega):
            seen.append((dms, j, k, omega))
            return G()

    class Opt:
        def apply_coeff_C_mat_CT(self, dm):
            return ('cart', dm.shape)

    opt = Opt()
    opt.mol = types.SimpleNamespace(nao=3, omega=-0.25)
    opt._jk_b200 = Plan()
    out = eb._jk_energy_per_atom(opt, np.zeros((2, 3, 3)), 1.0, 0.3)
    assert out.shape == (2, 3)
    assert seen == [(('cart', (2, 3, 3)), 1.0, 0.3, -0.25)]

