"""ctypes wrapper of the CPU oracle (jk_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by bench.py's CPU-baseline leg, as the checker.  The product package never
imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, '_build', 'libjk_oracle.so')

_lib = None


def build() -> str:
    subprocess.run(['make', '-s', '-C', HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.oracle_rys.argtypes = [ctypes.c_int, ctypes.c_double, dp, dp]
        L.oracle_eri_shells.argtypes = [ip, ip, dp, ctypes.c_int, ctypes.c_int,
                                        ctypes.c_int, ctypes.c_int, dp]
        L.oracle_q_cond.argtypes = [ip, ip, ctypes.c_int, dp, dp]
        L.oracle_jk.argtypes = [ip, ip, ctypes.c_int, dp, ip, dp, ctypes.c_int,
                                ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                dp, dp, ctypes.c_int,
                                ctypes.POINTER(ctypes.c_longlong)]
        L.oracle_jk_sample.argtypes = L.oracle_jk.argtypes + [
            ctypes.POINTER(ctypes.c_longlong), ctypes.c_longlong]
        L.oracle_eri_shells_rs.argtypes = [ip, ip, dp, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_int, ctypes.c_double, dp]
        L.oracle_jk_rs.argtypes = L.oracle_jk.argtypes + [ctypes.c_double]
        _lib = L
    return _lib


def _p(a, t=ctypes.c_double):
    return a.ctypes.data_as(ctypes.POINTER(t))


def _arrays(mol):
    atm = np.ascontiguousarray(mol._atm, dtype=np.int32)
    bas = np.ascontiguousarray(mol._bas, dtype=np.int32)
    env = np.ascontiguousarray(mol._env, dtype=np.float64)
    return atm, bas, env


def rys(n: int, x: float):
    r = np.zeros(n)
    w = np.zeros(n)
    if lib().oracle_rys(n, float(x), _p(r), _p(w)):
        raise ValueError('bad Rys order')
    return r, w


def eri_shells(mol, i, j, k, l, omega=0.0):
    """(ij|kl) of four shells; omega > 0: the long-range erf(omega r)/r."""
    from electrolites_b200.gto import ncart
    atm, bas, env = _arrays(mol)
    ls = [int(mol._bas[s, 1]) for s in (i, j, k, l)]
    out = np.zeros([ncart(x) for x in ls])
    if lib().oracle_eri_shells_rs(_p(atm, ctypes.c_int), _p(bas, ctypes.c_int),
                                  _p(env), i, j, k, l, float(omega), _p(out)):
        raise ValueError('unsupported shell')
    return out


def q_cond(mol):
    atm, bas, env = _arrays(mol)
    q = np.zeros((mol.nbas, mol.nbas))
    lib().oracle_q_cond(_p(atm, ctypes.c_int), _p(bas, ctypes.c_int),
                        mol.nbas, _p(env), _p(q))
    return q


def jk(mol, dms, tol=1e-13, with_j=True, with_k=True, nthreads=0, omega=0.0):
    """(vj, vk, n_quartets) for Cartesian-AO densities dms (n_dm, nao, nao);
    tol <= 0 disables screening; omega > 0: the long-range erf(omega r)/r."""
    atm, bas, env = _arrays(mol)
    dms = np.ascontiguousarray(dms, dtype=np.float64)
    squeeze = dms.ndim == 2
    if squeeze:
        dms = dms[None]
    ao_loc = np.ascontiguousarray(mol.ao_loc_nr(cart=True), dtype=np.int32)
    vj = np.zeros_like(dms)
    vk = np.zeros_like(dms)
    nq = ctypes.c_longlong(0)
    err = lib().oracle_jk_rs(_p(atm, ctypes.c_int), _p(bas, ctypes.c_int),
                             mol.nbas, _p(env), _p(ao_loc, ctypes.c_int),
                             _p(dms), dms.shape[0], float(tol), int(with_j),
                             int(with_k), _p(vj), _p(vk), int(nthreads),
                             ctypes.byref(nq), float(omega))
    if err:
        raise RuntimeError(f'oracle_jk failed ({err})')
    if squeeze:
        vj, vk = vj[0], vk[0]
    return vj, vk, nq.value


def jk_sample(mol, dms, ij_list, tol=1e-13, with_j=True, with_k=True, nthreads=0):
    """oracle J/K restricted to the bra shell pairs ij_list (linear index
    i*(i+1)/2 + j); returns (vj, vk, n_quartets)."""
    atm, bas, env = _arrays(mol)
    dms = np.ascontiguousarray(dms, dtype=np.float64)
    if dms.ndim == 2:
        dms = dms[None]
    ao_loc = np.ascontiguousarray(mol.ao_loc_nr(cart=True), dtype=np.int32)
    ij = np.ascontiguousarray(ij_list, dtype=np.int64)
    vj = np.zeros_like(dms)
    vk = np.zeros_like(dms)
    nq = ctypes.c_longlong(0)
    err = lib().oracle_jk_sample(
        _p(atm, ctypes.c_int), _p(bas, ctypes.c_int), mol.nbas, _p(env),
        _p(ao_loc, ctypes.c_int), _p(dms), dms.shape[0], float(tol), int(with_j),
        int(with_k), _p(vj), _p(vk), int(nthreads), ctypes.byref(nq),
        _p(ij, ctypes.c_longlong), len(ij))
    if err:
        raise RuntimeError(f'oracle_jk_sample failed ({err})')
    return vj, vk, nq.value


# ---------------------------------------------------------------------------
# fast FP64 checker (jk_check.c): same arithmetic, double-precision roots from
# Chebyshev fits of the long-double solver, OpenMP over bra pairs
# ---------------------------------------------------------------------------
def _check_lib():
    L = lib()
    if not getattr(L, '_check_ready', False):
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.check_rys.argtypes = [ctypes.c_int, ctypes.c_double, dp, dp]
        L.check_jk.argtypes = [ip, ip, ctypes.c_int, dp, ip, dp, ctypes.c_int,
                               ctypes.c_double, ctypes.c_int, ctypes.c_int, dp, dp,
                               ctypes.c_int, ctypes.POINTER(ctypes.c_longlong),
                               ctypes.c_double, ctypes.c_int, ctypes.c_int, dp]
        L.check_eri_shells.argtypes = [ip, ip, ctypes.c_int, dp, ip, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_double, dp]
        L._check_ready = True
    return L


def check_rys(n: int, x: float):
    r = np.zeros(n)
    w = np.zeros(n)
    if _check_lib().check_rys(n, float(x), _p(r), _p(w)):
        raise ValueError('bad Rys order or argument')
    return r, w


def check_eri_shells(mol, i, j, k, l, omega=0.0):
    """(ij|kl) of four shells (i >= j, k >= l) through the fast checker."""
    from electrolites_b200.gto import ncart
    atm, bas, env = _arrays(mol)
    ao_loc = np.ascontiguousarray(mol.ao_loc_nr(cart=True), dtype=np.int32)
    ls = [int(mol._bas[s, 1]) for s in (i, j, k, l)]
    out = np.zeros([ncart(x) for x in ls])
    if _check_lib().check_eri_shells(_p(atm, ctypes.c_int), _p(bas, ctypes.c_int), mol.nbas,
                                     _p(env), _p(ao_loc, ctypes.c_int), i, j, k, l,
                                     float(omega), _p(out)):
        raise ValueError('unsupported shell quartet')
    return out


def jk_fast(mol, dms, tol=1e-13, with_j=True, with_k=True, nthreads=0, omega=0.0,
            shard=0, nshard=1, want_q=False):
    """(vj, vk, n_quartets[, q_cond]) from the fast FP64 checker: the same
    quartets and contractions as jk(), restricted to bra shell pairs of shard
    `shard` of `nshard` (the shards sum to the full build)."""
    atm, bas, env = _arrays(mol)
    dms = np.ascontiguousarray(dms, dtype=np.float64)
    squeeze = dms.ndim == 2
    if squeeze:
        dms = dms[None]
    ao_loc = np.ascontiguousarray(mol.ao_loc_nr(cart=True), dtype=np.int32)
    vj = np.zeros_like(dms) if with_j else None
    vk = np.zeros_like(dms) if with_k else None
    q = np.zeros((mol.nbas, mol.nbas)) if want_q else None
    nq = ctypes.c_longlong(0)
    null = ctypes.POINTER(ctypes.c_double)()
    err = _check_lib().check_jk(
        _p(atm, ctypes.c_int), _p(bas, ctypes.c_int), mol.nbas, _p(env),
        _p(ao_loc, ctypes.c_int), _p(dms), dms.shape[0], float(tol), int(with_j),
        int(with_k), _p(vj) if with_j else null, _p(vk) if with_k else null,
        int(nthreads), ctypes.byref(nq), float(omega), int(shard), int(nshard),
        _p(q) if want_q else null)
    if err:
        raise RuntimeError(f'check_jk failed ({err})')
    if vj is None:
        vj = np.zeros_like(dms)
    if vk is None:
        vk = np.zeros_like(dms)
    if squeeze:
        vj, vk = vj[0], vk[0]
    return (vj, vk, nq.value, q) if want_q else (vj, vk, nq.value)


def grad_jk_fast(mol, dms, j_factor=1.0, k_factor=1.0, tol=1e-13, nthreads=0, omega=0.0):
    """(grad[natm, 3], n_quartets): dE/dR per atom of
    E = j/2 Tr[Dt J[Dt]] - k c sum_s Tr[D_s K[D_s]] (Dt = sum_s D_s, c = 1/4 for
    one density, 1/2 for two), densities symmetric and fixed in the AO basis,
    from the checker's analytic derivative integrals."""
    atm, bas, env = _arrays(mol)
    dms = np.ascontiguousarray(dms, dtype=np.float64)
    if dms.ndim == 2:
        dms = dms[None]
    ao_loc = np.ascontiguousarray(mol.ao_loc_nr(cart=True), dtype=np.int32)
    L = _check_lib()
    if not getattr(L, '_grad_ready', False):
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.check_grad_jk.argtypes = [ip, ctypes.c_int, ip, ctypes.c_int, dp, ip, dp, ctypes.c_int,
                                    ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_int, dp,
                                    ctypes.POINTER(ctypes.c_longlong)]
        L._grad_ready = True
    g = np.zeros((mol.natm, 3))
    nq = ctypes.c_longlong(0)
    err = L.check_grad_jk(_p(atm, ctypes.c_int), mol.natm, _p(bas, ctypes.c_int), mol.nbas,
                          _p(env), _p(ao_loc, ctypes.c_int), _p(dms), dms.shape[0], float(tol),
                          float(j_factor), float(k_factor), float(omega), int(nthreads), _p(g),
                          ctypes.byref(nq))
    if err:
        raise RuntimeError(f'check_grad_jk failed ({err})')
    return g, nq.value


def jk_energy(mol, dms, j_factor=1.0, k_factor=1.0, tol=1e-13, omega=0.0):
    """E = j/2 Tr[Dt J[Dt]] - k c sum_s Tr[D_s K[D_s]] from the checker's J/K."""
    dms = np.asarray(dms, dtype=np.float64)
    if dms.ndim == 2:
        dms = dms[None]
    vj, vk, _ = jk_fast(mol, dms, tol=tol, omega=omega)
    dt = dms.sum(axis=0)
    c = 0.25 if dms.shape[0] == 1 else 0.5
    ej = 0.5 * np.einsum('ij,ji->', dt, vj.sum(axis=0))
    ek = sum(np.einsum('ij,ji->', dms[s], vk[s]) for s in range(dms.shape[0]))
    return j_factor * ej - k_factor * c * ek
