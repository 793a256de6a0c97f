"""The allocation-free build entry point, jk_build_noalloc.

Callers that cannot let a library allocate device memory -- an SCF code that
gives all of it to its own caching pool, a latency-critical serving loop where
cudaMalloc/cudaFree would synchronise the device -- call jk_build_noalloc,
which takes its scratch from a fixed array inside the library instead of
allocating.  These tests call it through the C ABI and compare it with the
ordinary entry point, jk_build, on the same densities: as the first build of
a fresh plan, twice in a row (the second call runs on scratch the first one
left behind), alternating with jk_build on one plan, for J-only and K-only
requests, and with the device's free memory unchanged across the calls.

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


def _build(entry, opt, dms, hermi, torch, with_j=1, with_k=1, out=None):
    vj, vk = out if out is not None else (torch.zeros_like(dms), torch.zeros_like(dms))
    stream = torch.cuda.current_stream()
    _lib.check(entry(opt.plan, _vp(dms), dms.shape[0], hermi, with_j, with_k,
                     _vp(vj if with_j else None), _vp(vk if with_k else None), 0.0,
                     ctypes.c_void_p(stream.cuda_stream)), entry.__name__)
    _lib.check(_lib.lib().jk_sync(opt.plan, ctypes.c_void_p(stream.cuda_stream)), 'jk_sync')
    return vj, vk


def _inputs(torch, hermi, seed=7):
    mol = clusters.water_mole(4, 6.0, 31, basis='6-31g*')
    rng = np.random.default_rng(seed)
    D = clusters.atomic_density(mol, 3)
    dms = np.stack([D, D + 1e-2 * rng.standard_normal(D.shape)])
    if hermi == 1:
        dms = 0.5 * (dms + dms.transpose(0, 2, 1))
    return mol, torch.as_tensor(dms, device='cuda')


def _free_bytes(torch):
    torch.cuda.synchronize()
    free, _ = torch.cuda.mem_get_info()
    return free


@pytest.mark.parametrize('hermi', [1, 0])
def test_noalloc_first_build_then_twice_more(torch, hermi):
    """jk_build_noalloc as the first build of a fresh plan, then twice more,
    against jk_build on a second plan of the same molecule; the later calls
    leave the device's free memory unchanged."""
    from electrolites_b200.jk import VHFOpt
    mol, dms = _inputs(torch, hermi)
    L = _lib.lib()
    opt = VHFOpt(mol, 1e-13).build()
    first = _build(L.jk_build_noalloc, opt, dms, hermi, torch)
    ref = VHFOpt(mol, 1e-13).build()
    rj, rk = _build(L.jk_build, ref, dms, hermi, torch)
    assert float((first[0] - rj).abs().max()) <= ATOL
    assert float((first[1] - rk).abs().max()) <= ATOL
    out = (torch.zeros_like(dms), torch.zeros_like(dms))
    free0 = _free_bytes(torch)
    for _ in range(2):
        gj, gk = _build(L.jk_build_noalloc, opt, dms, hermi, torch, out=out)
        assert float((gj - rj).abs().max()) <= ATOL
        assert float((gk - rk).abs().max()) <= ATOL
    assert _free_bytes(torch) == free0


def test_noalloc_alternates_with_jk_build(torch):
    """jk_build_noalloc -> jk_build -> jk_build_noalloc on one plan: each
    switch moves the build's scratch between the plan's workspace and the
    library's array, and the descriptors follow."""
    from electrolites_b200.jk import VHFOpt
    mol, dms = _inputs(torch, 1, seed=11)
    L = _lib.lib()
    opt = VHFOpt(mol, 1e-13).build()
    a = _build(L.jk_build_noalloc, opt, dms, 1, torch)
    b = _build(L.jk_build, opt, dms, 1, torch)
    c = _build(L.jk_build_noalloc, opt, dms, 1, torch)
    for x, y in ((a, b), (c, b)):
        assert float((x[0] - y[0]).abs().max()) <= ATOL
        assert float((x[1] - y[1]).abs().max()) <= ATOL


@pytest.mark.parametrize('with_j,with_k', [(1, 0), (0, 1)])
def test_noalloc_j_only_and_k_only(torch, with_j, with_k):
    from electrolites_b200.jk import VHFOpt
    mol, dms = _inputs(torch, 1, seed=13)
    L = _lib.lib()
    opt = VHFOpt(mol, 1e-13).build()
    ref = VHFOpt(mol, 1e-13).build()
    for _ in range(2):
        gj, gk = _build(L.jk_build_noalloc, opt, dms, 1, torch, with_j, with_k)
        rj, rk = _build(L.jk_build, ref, dms, 1, torch, with_j, with_k)
        if with_j:
            assert float((gj - rj).abs().max()) <= ATOL
        if with_k:
            assert float((gk - rk).abs().max()) <= ATOL


def test_noalloc_rejects_builds_beyond_its_scratch(torch):
    """A build whose scratch exceeds the fixed array is refused with its own
    error code and a message, before any kernel runs; the ordinary entry
    point still works."""
    from electrolites_b200.jk import VHFOpt
    mol = clusters.water_mole(40, 11.0, 5, basis='6-31g*')      # 760 Cartesian AOs
    opt = VHFOpt(mol, 1e-13).build()
    dms = torch.zeros((2, mol.nao_cart, mol.nao_cart), dtype=torch.float64, device='cuda')
    vj = torch.empty_like(dms)
    vk = torch.empty_like(dms)
    L = _lib.lib()
    rc = L.jk_build_noalloc(opt.plan, _vp(dms), 2, 1, 1, 1, _vp(vj), _vp(vk), 0.0, None)
    assert rc == 7                  # JK_ERR_SCRATCH
    assert b'static scratch' in L.jk_last_error()
    gj, gk = _build(L.jk_build, opt, dms, 1, torch)
    assert float(gj.abs().max()) == 0.0 and float(gk.abs().max()) == 0.0
