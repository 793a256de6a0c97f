"""The McMurchie-Davidson J kernel (J-only builds) against the oracle and
against the Rys J engine, through the C ABI.

The reference's own J tests compare its MD kernels with GPU4PySCF's
MD_build_j at 1e-12 relative over several density counts (tests/test_j_ndm.py
there).  Here: every class that has an MD kernel (l_i + l_j + l_k + l_l <= 6)
forced on, on the all-class molecule and water clusters, one and two
densities, each J element within 1e-10 of the oracle's J-only build; a
three-density build (beyond the MD kernel's two) and the long-range operator
keep the Rys J engine and stay exact; the MD and Rys builds of one plan agree
to 1e-11.
"""
import numpy as np
import pytest

from electrolites_b200 import clusters
from electrolites_b200.gto import Mole

pytestmark = pytest.mark.gpu

ATOL = 1e-10
TOL = 1e-13


@pytest.fixture(scope='module')
def torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return torch


def all_class_mol():
    b = {
        'H': [[0, (1.3, 0.6), (0.3, 0.5)], [1, (0.9, 1.0)], [2, (0.7, 1.0)], [3, (0.6, 1.0)]],
        'He': [[0, (0.8, 1.0)], [1, (1.4, 0.7), (0.4, 0.4)], [2, (1.1, 1.0)], [3, (0.9, 1.0)]],
        'C': [[0, (2.1, 1.0)], [1, (0.5, 1.0)], [2, (0.9, 0.5), (0.35, 0.6)], [3, (1.2, 1.0)]],
    }
    atom = [('H', (0.0, 0.0, 0.0)), ('He', (0.9, 0.3, -0.4)), ('C', (-0.5, 1.1, 0.6))]
    return Mole(atom, basis=b, cart=True)


def _dms(mol, n_dm, seed):
    rng = np.random.default_rng(seed)
    D = clusters.atomic_density(mol, seed) + 0.02 * rng.standard_normal((mol.nao_cart,) * 2)
    D = 0.5 * (D + D.T)
    return clusters.density_stack(D, n_dm, seed + 1, 0.05)


@pytest.mark.parametrize('name,n_dm', [('spdf', 1), ('spdf', 2), ('h2o4_631gs', 2),
                                       ('h2o2_tzvp', 1)])
def test_md_j_matches_oracle(oracle, torch, name, n_dm):
    from electrolites_b200.jk import VHFOpt
    mol = {'spdf': all_class_mol,
           'h2o4_631gs': lambda: clusters.water_mole(4, 5.0, 41, basis='6-31g*'),
           'h2o2_tzvp': lambda: clusters.water_mole(2, 4.0, 42, basis='def2-tzvp')}[name]()
    dms = _dms(mol, n_dm, 7)
    opt = VHFOpt(mol, TOL).build()
    opt.set_jmd(1)
    vj = opt.get_j(torch.as_tensor(dms)).cpu().numpy()
    rj, _, _ = oracle.jk(mol, dms, tol=TOL, with_j=True, with_k=False)
    assert np.abs(vj - rj).max() <= ATOL
    opt.set_jmd(0)
    vr = opt.get_j(torch.as_tensor(dms)).cpu().numpy()
    assert np.abs(vj - vr).max() <= 1e-11


def test_md_j_leaves_other_builds_to_the_rys_engine(oracle, torch):
    """Three densities, and the long-range operator: the MD kernel does not
    serve them; J stays exact with it switched on."""
    from electrolites_b200.jk import VHFOpt
    mol = all_class_mol()
    opt = VHFOpt(mol, TOL).build()
    opt.set_jmd(1)
    dms = _dms(mol, 3, 9)
    vj = opt.get_j(torch.as_tensor(dms)).cpu().numpy()
    rj, _, _ = oracle.jk(mol, dms, tol=TOL, with_j=True, with_k=False)
    assert np.abs(vj - rj).max() <= ATOL
    d2 = dms[:2]
    vl, _ = opt.get_jk(torch.as_tensor(d2), hermi=1, with_k=False, omega=0.4)
    rl, _, _ = oracle.jk(mol, d2, tol=TOL, with_j=True, with_k=False, omega=0.4)
    assert np.abs(vl.cpu().numpy() - rl).max() <= ATOL


def test_md_j_class_switch(torch):
    from electrolites_b200 import _lib
    from electrolites_b200.jk import VHFOpt, class_keys
    mol = clusters.water_mole(1, 3.0, 7, basis='6-31g*')
    opt = VHFOpt(mol, TOL).build()
    keys = class_keys()
    big = keys.index((3, 3, 3, 3))
    with pytest.raises(_lib.JKError):
        opt.set_jmd(1, big)          # (ff|ff): no MD kernel
    opt.set_jmd(1, keys.index((1, 0, 0, 0)))
    opt.set_jmd(-1)
