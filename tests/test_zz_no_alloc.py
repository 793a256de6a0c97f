"""The allocation-free build entry point, jk_build_noalloc.

Callers that cannot let a library allocate device memory -- an SCF code that
gives all of it to its own caching pool, a latency-critical serving loop where
cudaMalloc/cudaFree would synchronise the device -- call jk_build_noalloc,
which takes its scratch from a fixed array inside the library instead of
allocating.  These tests call it through the C ABI and compare it with the
ordinary entry point, jk_build, on the same plan and densities, twice in a
row (the second call runs on scratch the first one left behind).

The file is named so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

from electrolites_b200 import _lib, clusters

pytestmark = pytest.mark.gpu

ATOL = 1e-10        # the parity tolerance of the J/K tests


@pytest.fixture(scope='module')
def torch():
    import torch
    if not torch.cuda.is_available():
        pytest.skip('no CUDA device')
    return torch


def _vp(t):
    return ctypes.c_void_p(t.data_ptr() if t is not None else 0)


def _build(entry, opt, dms, hermi, torch):
    vj = torch.zeros_like(dms)
    vk = torch.zeros_like(dms)
    stream = torch.cuda.current_stream()
    _lib.check(entry(opt.plan, _vp(dms), dms.shape[0], hermi, 1, 1, _vp(vj), _vp(vk), 0.0,
                     ctypes.c_void_p(stream.cuda_stream)), entry.__name__)
    _lib.check(_lib.lib().jk_sync(opt.plan, ctypes.c_void_p(stream.cuda_stream)), 'jk_sync')
    return vj, vk


@pytest.mark.parametrize('hermi', [1, 0])
def test_noalloc_matches_jk_build_twice(torch, hermi):
    from electrolites_b200.jk import VHFOpt
    mol = clusters.water_mole(4, 6.0, 31, basis='6-31g*')
    opt = VHFOpt(mol, 1e-13).build()
    rng = np.random.default_rng(7)
    D = clusters.atomic_density(mol, 3)
    dms = np.stack([D, D + 1e-2 * rng.standard_normal(D.shape)])
    if hermi == 1:
        dms = 0.5 * (dms + dms.transpose(0, 2, 1))
    dms = torch.as_tensor(dms, device='cuda')
    L = _lib.lib()
    rj, rk = _build(L.jk_build, opt, dms, hermi, torch)
    for _ in range(2):
        gj, gk = _build(L.jk_build_noalloc, opt, dms, hermi, torch)
        assert float((gj - rj).abs().max()) <= ATOL
        assert float((gk - rk).abs().max()) <= ATOL


def test_noalloc_rejects_builds_beyond_its_scratch(torch):
    """A build whose scratch exceeds the fixed array is refused with a
    message, before any kernel runs; the ordinary entry point still works."""
    from electrolites_b200.jk import VHFOpt
    mol = clusters.water_mole(40, 11.0, 5, basis='6-31g*')      # 760 Cartesian AOs
    opt = VHFOpt(mol, 1e-13).build()
    dms = torch.zeros((2, mol.nao_cart, mol.nao_cart), dtype=torch.float64, device='cuda')
    vj = torch.empty_like(dms)
    vk = torch.empty_like(dms)
    L = _lib.lib()
    rc = L.jk_build_noalloc(opt.plan, _vp(dms), 2, 1, 1, 1, _vp(vj), _vp(vk), 0.0, None)
    assert rc == 5
    assert b'static scratch' in L.jk_last_error()
