"""The engine's nuclear gradient of the two-electron energy (jk_grad, through
the C ABI) against the checker's analytic gradient.

The reference's own tests compare its gradient kernels with GPU4PySCF's at
1e-11 relative (tests/test_uejk.py there: closed shell and two spin
densities, (j, k) = (1, 0.2), (1, 0), (0, 0.25), bases up to g).  Here the
counterpart is oracle/jk_check.c's derivative integrals, themselves pinned to
finite differences of the checker's J/K energies (tests/test_check.py).
Tolerance: every force component within 1e-10 relative to the largest.
Cases: every class up to (ff|ff) in one molecule (both the per-lane form and
the per-warp form of the kernel), one and two densities, the three (j, k)
pairs above, the long-range and short-range operators, and water clusters in
6-31G* and def2-TZVP shapes; forces sum to zero.
"""
import numpy as np
import pytest

from electrolites_b200 import clusters
from electrolites_b200.gto import Mole

pytestmark = pytest.mark.gpu

RTOL = 1e-10
FACTORS = ((1.0, 0.2), (1.0, 0.0), (0.0, 0.25))


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


def noisy_density(mol, seed, noise=0.05):
    rng = np.random.default_rng(seed)
    D = clusters.atomic_density(mol, seed) + noise * rng.standard_normal((mol.nao_cart,) * 2)
    return 0.5 * (D + D.T)


def _check(got, ref):
    scale = max(np.abs(ref).max(), 1e-30)
    err = np.abs(got - ref).max() / scale
    assert err <= RTOL, err
    assert np.abs(got.sum(axis=0)).max() <= 1e-11 * max(1.0, scale)


@pytest.mark.parametrize('n_dm', [1, 2])
def test_gradient_every_class(oracle, torch, n_dm):
    from electrolites_b200.jk import VHFOpt
    mol = all_class_mol()
    D = noisy_density(mol, 3)
    dms = D[None] if n_dm == 1 else clusters.uhf_pair(D, 4, 0.05)
    opt = VHFOpt(mol, 1e-16).build()
    for jf, kf in FACTORS:
        got = opt.jk_energy_per_atom(torch.as_tensor(dms), jf, kf).cpu().numpy()
        ref, _ = oracle.grad_jk_fast(mol, dms, jf, kf, tol=0)
        _check(got, ref)


def test_gradient_range_separated(oracle, torch):
    """omega > 0: erf(omega r)/r; omega < 0: erfc(|omega| r)/r, the full
    minus the long-range gradient."""
    from electrolites_b200.jk import VHFOpt
    mol = all_class_mol()
    dms = clusters.uhf_pair(noisy_density(mol, 5), 6, 0.05)
    opt = VHFOpt(mol, 1e-16).build()
    lr = opt.jk_energy_per_atom(torch.as_tensor(dms), 1.0, 0.3, omega=0.4).cpu().numpy()
    ref_lr, _ = oracle.grad_jk_fast(mol, dms, 1.0, 0.3, tol=0, omega=0.4)
    _check(lr, ref_lr)
    sr = opt.jk_energy_per_atom(torch.as_tensor(dms), 1.0, 0.3, omega=-0.4).cpu().numpy()
    full, _ = oracle.grad_jk_fast(mol, dms, 1.0, 0.3, tol=0)
    _check(sr, full - ref_lr)


@pytest.mark.parametrize('name', ['h2o4_631gs', 'h2o2_tzvp'])
def test_gradient_water_clusters(oracle, torch, name):
    from electrolites_b200 import jk
    mol = {'h2o4_631gs': lambda: clusters.water_mole(4, 5.0, 31, basis='6-31g*'),
           'h2o2_tzvp': lambda: clusters.water_mole(2, 4.0, 32, basis='def2-tzvp')}[name]()
    D = noisy_density(mol, 7, 0.01)
    for dms in (D[None], clusters.uhf_pair(D, 8, 0.05)):
        opt = jk.VHFOpt(mol, 1e-14).build()
        got = jk.jk_energy_per_atom(mol, dms, 1.0, 0.2, vhfopt=opt)
        ref, _ = oracle.grad_jk_fast(mol, dms, 1.0, 0.2, tol=0)
        _check(got, ref)


def test_gradient_repeats_and_rejects_bad_arguments(torch):
    from electrolites_b200 import _lib
    from electrolites_b200.jk import VHFOpt
    mol = clusters.water_mole(1, 3.0, 7, basis='6-31g*')
    opt = VHFOpt(mol, 1e-13).build()
    dms = torch.as_tensor(clusters.uhf_pair(noisy_density(mol, 9), 10, 0.05))
    a = opt.jk_energy_per_atom(dms, 1.0, 0.2).cpu().numpy()
    b = opt.jk_energy_per_atom(dms, 1.0, 0.2).cpu().numpy()
    assert np.abs(a - b).max() <= 1e-13 * np.abs(a).max()
    with pytest.raises(ValueError):
        opt.jk_energy_per_atom(torch.cat([dms, dms[:1]]), 1.0, 0.2)
    with pytest.raises(_lib.JKError):
        opt.jk_energy_per_atom(dms, float('nan'), 0.2)
    # the plan still builds J/K after a gradient
    vj, vk = opt.get_jk(dms, hermi=1)
    assert torch.isfinite(vj).all() and torch.isfinite(vk).all()
