"""Drop-in J/K builds on the B200 engine.

Mirrors the interface the reference patches (electrolites/__init__.py:59-61,
107): GPU4PySCF's module functions ``jk.get_jk(mol, dm, hermi, vhfopt,
with_j, with_k, omega, verbose)``, ``jk.get_j`` and ``jk.get_k``, and the
option object's methods ``_VHFOpt.get_jk(dms, hermi, verbose)``,
``_VHFOpt.get_k(dms, hermi, verbose, omega, lr_factor, sr_factor)`` and
``j_engine._VHFOpt.get_j(dms, verbose)`` (electrolites/fastjk.py:276,
electrolites/fastk.py:642, electrolites/fastj.py:540).

Semantics kept from the reference:
  * ``dms`` is (n_dm, nao, nao) (or (nao, nao)); ``hermi`` 1 = symmetric,
    2 = antisymmetric (J is zero, K antisymmetric), 0 = general;
  * vj[k,l] = sum_ij (ij|kl) D[j,i], vk[i,l] = sum_jk (ij|kl) D[j,k];
  * quartets are screened with the direct-SCF threshold of the option
    object: kept when q_ij + q_kl + log max|D| > log(direct_scf_tol);
  * the operator follows PySCF's omega convention: omega = 0 (or None) the
    Coulomb operator 1/r, omega > 0 the long-range erf(omega r)/r, omega < 0
    the short-range erfc(|omega| r)/r = 1/r - erf(|omega| r)/r; ``get_k``'s
    lr_factor / sr_factor ask for lr K_lr + sr K_sr (GPU4PySCF 1.8's
    range-separated exchange), built as sr K_full + (lr - sr) K_lr in one
    fused pass (the reference's get_k_rsh, electrolites/fastk.py:774-899:
    the Rys quadrature runs once per operator inside the primitive loop,
    screening by the Coulomb bound and the digest are shared).  The
    reference serves the full and long-range operators and hands the
    short-range one back (electrolites/fastk.py:642-663,904-925); here all
    three run on the engine.

The option-object methods work in the Cartesian AO basis of the molecule
they were built for.  The module functions take densities in the
molecule's own AO basis (spherical unless ``mol.cart``) and transform them.
"""
from __future__ import annotations

import collections
import ctypes
import hashlib

import numpy as np

from . import _lib

DEFAULT_TOL = 1e-13


def _torch():
    import torch
    return torch


def _as_int32(a):
    return np.ascontiguousarray(np.asarray(a), dtype=np.int32)


class VHFOpt:
    """Plan of one molecule: shell pairs, primitive pairs, Schwarz bounds,
    pair lists by class, all resident on the device across builds.

    The counterpart of GPU4PySCF's ``jk._VHFOpt(mol, cutoff)``.
    """

    def __init__(self, mol, cutoff: float = DEFAULT_TOL, device: int | None = None):
        self.mol = mol
        self.direct_scf_tol = float(cutoff)
        self.device = device
        self._plan = None
        self.nao = None

    # ------------------------------------------------------------------
    def build(self):
        torch = _torch()
        if not torch.cuda.is_available():
            raise RuntimeError('the J/K engine needs a CUDA device')
        if self.device is None:
            self.device = torch.cuda.current_device()
        mol = self.mol
        self._atm = _as_int32(mol._atm)
        self._bas = _as_int32(mol._bas)
        self._env = np.ascontiguousarray(mol._env, dtype=np.float64)
        self._ao_loc = _as_int32(mol.ao_loc_nr(cart=True))
        plan = ctypes.c_void_p()
        L = _lib.lib()
        _lib.check(L.jk_plan_create(
            self._atm.ctypes.data, len(self._atm), self._bas.ctypes.data,
            len(self._bas), self._env.ctypes.data, self._ao_loc.ctypes.data,
            self.direct_scf_tol, int(self.device), ctypes.byref(plan)),
            'jk_plan_create')
        self._plan = plan
        nao = ctypes.c_int()
        npairs = ctypes.c_longlong()
        _lib.check(L.jk_plan_info(plan, ctypes.byref(nao), ctypes.byref(npairs)),
                   'jk_plan_info')
        self.nao = nao.value
        self.npairs = npairs.value
        self._plan_tol = self._applied_tol = self.direct_scf_tol
        from . import autotune
        table = autotune.load(self.device, 'single')
        if table:
            autotune.apply(self, table)
        return self

    def __del__(self):
        try:
            if self._plan is not None:
                _lib.lib().jk_plan_destroy(self._plan)
                self._plan = None
        except Exception:
            pass

    @property
    def plan(self):
        if self._plan is None:
            self.build()
        return self._plan

    def set_jengine(self, on=True):
        """J-only builds through the J engine (default) or the (ij|kl)
        digest of J/K builds; the same J to rounding."""
        _lib.check(_lib.lib().jk_plan_set_jengine(self.plan, int(bool(on))),
                   'jk_plan_set_jengine')

    def apply_tol(self):
        """Hands ``direct_scf_tol`` to the plan if it changed since the last
        build: builds read it at call time, as the reference's do.  A value
        below the threshold the plan was built with is an error (its pair
        lists lack the pairs a tighter screen needs)."""
        plan = self.plan
        tol = float(self.direct_scf_tol)
        if tol != self._applied_tol:
            _lib.check(_lib.lib().jk_plan_set_tol(plan, tol), 'jk_plan_set_tol')
            self._applied_tol = tol
        return plan

    # ------------------------------------------------------------------
    def _prepare(self, dms):
        torch = _torch()
        if callable(dms):
            dms = dms()
        if not isinstance(dms, torch.Tensor):
            dms = torch.as_tensor(dms)
        squeeze = dms.ndim == 2
        if squeeze:
            dms = dms[None]
        if dms.ndim != 3 or dms.shape[-1] != self.nao or dms.shape[-2] != self.nao:
            raise ValueError(f'dms must be (n_dm, {self.nao}, {self.nao}); got '
                             f'{tuple(dms.shape)}')
        dev = torch.device('cuda', self.device)
        dms = dms.to(device=dev, dtype=torch.float64).contiguous()
        return dms, squeeze

    def build_jk_async(self, dms, hermi=1, with_j=True, with_k=True,
                       vj=None, vk=None, mixed_threshold=0.0, stream=None, omega=0.0,
                       terms=None):
        """Enqueue one build on ``stream`` (torch's current stream by default)
        without synchronising; dms must be a contiguous float64 CUDA tensor
        (n_dm, nao, nao).  The operator is ``terms`` = [(c_t, omega_t >= 0)],
        one or two of them, sum_t c_t op(omega_t) in one pass (op(0) = 1/r,
        op(w > 0) = erf(w r)/r); without terms, op(omega).  Returns (vj, vk)."""
        torch = _torch()
        plan = self.apply_tol()
        n = dms.shape[0]
        if terms is None:
            terms = [(1.0, float(omega))]
        if not 1 <= len(terms) <= 2:
            raise ValueError('the operator takes one or two terms')
        coef = (ctypes.c_double * 2)(*[float(c) for c, _ in terms], *([0.0] * (2 - len(terms))))
        om = (ctypes.c_double * 2)(*[float(w) for _, w in terms], *([0.0] * (2 - len(terms))))
        if with_j and vj is None:
            vj = torch.empty_like(dms)
        if with_k and vk is None:
            vk = torch.empty_like(dms)
        if stream is None:
            stream = torch.cuda.current_stream(dms.device)
        _lib.check(_lib.lib().jk_build_op(
            plan, ctypes.c_void_p(dms.data_ptr()), n, int(hermi), int(bool(with_j)),
            int(bool(with_k)), ctypes.c_void_p(vj.data_ptr() if with_j else 0),
            ctypes.c_void_p(vk.data_ptr() if with_k else 0), float(mixed_threshold),
            len(terms), ctypes.cast(coef, ctypes.c_void_p), ctypes.cast(om, ctypes.c_void_p),
            ctypes.c_void_p(stream.cuda_stream)), 'jk_build_op')
        return vj, vk

    def sync(self, stream=None):
        torch = _torch()
        if stream is None:
            stream = torch.cuda.current_stream(torch.device('cuda', self.device))
        _lib.check(_lib.lib().jk_sync(self.plan, ctypes.c_void_p(stream.cuda_stream)),
                   'jk_sync')

    def _combo(self, dms, hermi, with_j, with_k, mixed_threshold, terms):
        """(vj, vk) of the operator sum_t c_t op(omega_t) over terms
        [(c_t, omega_t >= 0)], one fused build."""
        vj, vk = self.build_jk_async(dms, hermi, with_j, with_k,
                                     mixed_threshold=mixed_threshold, terms=terms)
        self.sync()
        return vj, vk

    def get_jk(self, dms, hermi=1, verbose=None, with_j=True, with_k=True,
               mixed_threshold=0.0, omega=None):
        """(vj, vk) as CUDA tensors shaped like dms (Cartesian AO basis), for
        the operator of ``omega`` (PySCF's convention, see the module notes)."""
        dms, squeeze = self._prepare(dms)
        vj, vk = self._combo(dms, hermi, with_j, with_k, mixed_threshold,
                             _rsh_terms(omega, None, None))
        if squeeze:
            vj = vj[0] if vj is not None else None
            vk = vk[0] if vk is not None else None
        return vj, vk

    def get_k(self, dms, hermi=1, verbose=None, omega=None, lr_factor=None,
              sr_factor=None):
        """K for lr_factor K_lr + sr_factor K_sr at omega (factors absent: the
        operator of omega alone)."""
        dms, squeeze = self._prepare(dms)
        _, vk = self._combo(dms, hermi, False, True, 0.0,
                            _rsh_terms(omega, lr_factor, sr_factor))
        return vk[0] if squeeze else vk

    def get_j(self, dms, verbose=None, hermi=1):
        vj, _ = self.get_jk(dms, hermi, verbose, with_j=True, with_k=False)
        return vj

    def jk_energy_per_atom(self, dms, j_factor=1.0, k_factor=1.0, omega=0.0, stream=None):
        """Per-atom nuclear gradient, a (natm, 3) float64 CUDA tensor, of
        E = j/2 Tr[Dt J[Dt]] - k c sum_s Tr[D_s K[D_s]] for one or two
        symmetric densities dms (plan's Cartesian basis, held fixed in it),
        Dt = sum_s D_s, c = 1/4 for one density and 1/2 for two -- what
        GPU4PySCF's grad.rhf._jk_energy_per_atom returns and the reference's
        fastejk replaces (electrolites/fastejk.py:270-356, its factors at
        :308-316).  omega > 0: the long-range operator erf(omega r)/r;
        omega < 0: the short-range one, as the full minus the long-range
        gradient (two passes)."""
        torch = _torch()
        dms, _ = self._prepare(dms)
        n = dms.shape[0]
        if n not in (1, 2):
            raise ValueError(f'jk_energy_per_atom takes one or two densities; got {n}')
        omega = 0.0 if omega is None else float(omega)
        plan = self.apply_tol()
        if stream is None:
            stream = torch.cuda.current_stream(dms.device)
        natm = len(self._atm)

        def one(w):
            out = torch.empty((natm, 3), dtype=torch.float64, device=dms.device)
            _lib.check(_lib.lib().jk_grad(
                plan, ctypes.c_void_p(dms.data_ptr()), n, float(j_factor), float(k_factor),
                float(w), ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream.cuda_stream)),
                'jk_grad')
            return out

        if omega >= 0:
            g = one(omega)
        else:
            g = one(0.0)
            g -= one(-omega)
        self.sync(stream)
        return g

    def class_counts(self, with_f32=False):
        """{(li, lj, lk, ll): (quartets, primitive quartets)} evaluated by the
        last build; with_f32 appends the quartets evaluated in FP32."""
        L = _lib.lib()
        ncls = ctypes.c_int()
        _lib.check(L.jk_last_counts(self.plan, None, None, None, 0, ctypes.byref(ncls)),
                   'jk_last_counts')
        q = (ctypes.c_ulonglong * ncls.value)()
        pq = (ctypes.c_ulonglong * ncls.value)()
        q32 = (ctypes.c_ulonglong * ncls.value)()
        _lib.check(L.jk_last_counts(self.plan, q, pq, q32, ncls.value, ctypes.byref(ncls)),
                   'jk_last_counts')
        out = {}
        for k in range(ncls.value):
            ls = [ctypes.c_int() for _ in range(5)]
            _lib.check(L.jk_class_info(k, *[ctypes.byref(x) for x in ls]), 'jk_class_info')
            key = tuple(x.value for x in ls[:4])
            out[key] = (int(q[k]), int(pq[k])) + ((int(q32[k]),) if with_f32 else ())
        return out

    def set_timing(self, enable=True):
        """Per-class kernel events: True / 1 times each class alone (class
        kernels serialised on the build's stream), 2 records the events on
        the class streams of the default launch order, False / 0 none."""
        mode = 2 if enable == 2 else int(bool(enable))
        _lib.check(_lib.lib().jk_set_timing(self.plan, mode), 'jk_set_timing')

    def last_class_ms(self):
        """({(li, lj, lk, ll): ms of that class kernel in the last build},
        number of kernels the last build launched)."""
        L = _lib.lib()
        n = 64
        ms = (ctypes.c_float * n)()
        launches = ctypes.c_int()
        _lib.check(L.jk_last_class_ms(self.plan, ms, n, ctypes.byref(launches)),
                   'jk_last_class_ms')
        out = {}
        for k in range(n):
            ls = [ctypes.c_int() for _ in range(5)]
            if L.jk_class_info(k, *[ctypes.byref(x) for x in ls]) != 0:
                break
            if ms[k] > 0:
                out[tuple(x.value for x in ls[:4])] = float(ms[k])
        return out, launches.value

    def set_shard(self, rank: int, size: int):
        """Later builds evaluate only this rank's share of the task lists
        (tasks rank, rank + size, ...); the sum of vj / vk over the ranks is
        the full result (electrolites_b200.shard does the all-reduce)."""
        _lib.check(_lib.lib().jk_plan_set_shard(self.plan, int(rank), int(size)),
                   'jk_plan_set_shard')

    def set_jmd(self, mode: int = 1, cls: int = -1):
        """J-only builds: McMurchie-Davidson J kernel for class index cls
        (-1: every class that has one) on (1), off (0) or the class's
        default (-1)."""
        _lib.check(_lib.lib().jk_plan_set_jmd(self.plan, int(cls), int(mode)), 'jk_plan_set_jmd')

    def set_tuning(self, cls: int, tasks_per_sm: int, blocks_per_sm: int = 0, fp32: int = -1):
        """Per-class launch tuning (class index k of class_keys(); -1 resets
        every class)."""
        _lib.check(_lib.lib().jk_plan_set_tuning(self.plan, int(cls), int(tasks_per_sm),
                                                 int(blocks_per_sm), int(fp32)),
                   'jk_plan_set_tuning')

    def memory(self):
        """(bytes of the plan's resident tables, bytes of its build workspace)."""
        t = ctypes.c_longlong()
        w = ctypes.c_longlong()
        _lib.check(_lib.lib().jk_plan_memory(self.plan, ctypes.byref(t), ctypes.byref(w)),
                   'jk_plan_memory')
        return t.value, w.value

    def q_cond(self):
        nb = len(self._bas)
        q = np.zeros((nb, nb), dtype=np.float32)
        _lib.check(_lib.lib().jk_plan_q_cond(
            self.plan, q.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), nb),
            'jk_plan_q_cond')
        return q


def class_keys():
    """[(li, lj, lk, ll), ...] of the engine's classes, by class index."""
    L = _lib.lib()
    keys = []
    k = 0
    while True:
        ls = [ctypes.c_int() for _ in range(5)]
        if L.jk_class_info(k, *[ctypes.byref(x) for x in ls]) != 0:
            return keys
        keys.append(tuple(x.value for x in ls[:4]))
        k += 1


def _rsh_terms(omega, lr_factor, sr_factor):
    """[(coefficient, omega >= 0), ...] whose combination is the requested
    operator: lr K_erf(w) + sr K_erfc(w) = sr K_full + (lr - sr) K_erf(w),
    w = |omega|; without factors omega > 0 is (1, 0) and omega < 0 is (0, 1)."""
    om = float(omega or 0.0)
    if lr_factor is None and sr_factor is None:
        lr, sr = (1.0, 1.0) if om == 0 else ((1.0, 0.0) if om > 0 else (0.0, 1.0))
    else:
        lr = 1.0 if lr_factor is None else float(lr_factor)
        sr = 1.0 if sr_factor is None else float(sr_factor)
    w = abs(om)
    if w == 0:
        if lr != sr:
            raise ValueError('lr_factor != sr_factor needs omega != 0')
        return [(lr, 0.0)]
    terms = []
    if sr != 0:
        terms.append((sr, 0.0))
    if lr - sr != 0:
        terms.append((lr - sr, w))
    return terms or [(0.0, 0.0)]


# ----------------------------------------------------------------------
# module-level functions (GPU4PySCF's jk.get_jk / get_j / get_k)
# ----------------------------------------------------------------------
# plans of the module functions, keyed by the molecule's content (geometry,
# basis, AO layout and screening threshold), least recently used last out:
# a molecule moved in place (PySCF's set_geom_ defaults to inplace=True, as
# do scanners) gets a new plan, and the cache holds at most _OPTS_MAX plans
_OPTS = collections.OrderedDict()
_OPTS_MAX = 8


def _opt_key(mol):
    h = hashlib.sha1()
    for a, dt in ((mol._atm, np.int32), (mol._bas, np.int32), (mol._env, np.float64)):
        h.update(np.ascontiguousarray(a, dtype=dt).tobytes())
        h.update(b'|')
    h.update(np.ascontiguousarray(mol.ao_loc_nr(cart=True), dtype=np.int64).tobytes())
    tol = float(getattr(mol, 'direct_scf_tol', DEFAULT_TOL))
    return h.hexdigest(), tol


def _opt_for(mol, vhfopt):
    if vhfopt is not None:
        return vhfopt
    key = _opt_key(mol)
    opt = _OPTS.get(key)
    if opt is None:
        opt = VHFOpt(mol, key[1]).build()
        _OPTS[key] = opt
        while len(_OPTS) > _OPTS_MAX:
            _OPTS.popitem(last=False)
    else:
        _OPTS.move_to_end(key)
    return opt


def _to_cart(mol, dms):
    torch = _torch()
    if getattr(mol, 'cart', False):
        return dms, None
    c = torch.as_tensor(mol.cart2sph_coeff(), dtype=torch.float64, device=dms.device)
    return c @ dms @ c.T, c


def get_jk(mol, dm, hermi=1, vhfopt=None, with_j=True, with_k=True, omega=None,
           verbose=None):
    """(vj, vk) for densities in mol's AO basis.  numpy in -> numpy out;
    torch in -> torch out."""
    torch = _torch()
    was_numpy = not isinstance(dm, torch.Tensor) and not hasattr(dm, '__cuda_array_interface__')
    opt = _opt_for(mol, vhfopt)
    d = torch.as_tensor(np.asarray(dm) if was_numpy else dm)
    squeeze = d.ndim == 2
    if squeeze:
        d = d[None]
    d = d.to(device=torch.device('cuda', opt.device), dtype=torch.float64)
    dc, c = _to_cart(mol, d)
    vj, vk = opt.get_jk(dc.contiguous(), hermi, verbose, with_j, with_k, omega=omega)
    outs = []
    for v in (vj, vk):
        if v is None:
            outs.append(None)
            continue
        if c is not None:
            v = c.T @ v @ c
        if squeeze:
            v = v[0]
        outs.append(v.cpu().numpy() if was_numpy else v)
    return tuple(outs)


def jk_energy_per_atom(mol, dm, j_factor=1.0, k_factor=1.0, vhfopt=None, omega=None):
    """VHFOpt.jk_energy_per_atom for densities in mol's AO basis (one
    (nao, nao) or a stack of two); returns a numpy (natm, 3) array."""
    torch = _torch()
    opt = _opt_for(mol, vhfopt)
    d = torch.as_tensor(dm)
    if d.ndim == 2:
        d = d[None]
    d = d.to(device=torch.device('cuda', opt.device), dtype=torch.float64)
    dc, _ = _to_cart(mol, d)
    if omega is None:
        omega = float(getattr(mol, 'omega', 0.0) or 0.0)
    g = opt.jk_energy_per_atom(dc.contiguous(), j_factor, k_factor, omega)
    return g.cpu().numpy()


def get_j(mol, dm, hermi=1, vhfopt=None, verbose=None):
    return get_jk(mol, dm, hermi, vhfopt, True, False, None, verbose)[0]


def get_k(mol, dm, hermi=1, vhfopt=None, omega=None, verbose=None):
    return get_jk(mol, dm, hermi, vhfopt, False, True, omega, verbose)[1]
