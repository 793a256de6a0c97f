"""Batched J/K builds: many molecules in one launch stream.

``JKBatch.build`` computes J and/or K for a list of molecules -- each a
``VHFOpt`` plan with its own stack of densities -- as one persistent kernel
per angular-momentum class over the task lists of every molecule, instead of
one launch sequence per molecule.  With ``use_graph=True`` the launch stream
is captured in a CUDA graph on the second call and replayed by every later
call with the same plans and buffers, so an SCF loop (or a serving cycle)
over a fixed set of molecules writes new density values into the same
tensors and replays.

The results equal one ``VHFOpt.get_jk`` per molecule with the same
arguments (hermi, with_j, with_k, mixed_threshold apply to every molecule).
The reference builds one molecule per call (electrolites/fastjk.py:276,
electrolites/fastk.py:642); this is the batched form of that call.
"""
from __future__ import annotations

import ctypes

from . import _lib
from .jk import class_keys


def _torch():
    import torch
    return torch


class JKBatch:
    """A batch engine on one device: task rows, descriptors, workspace and
    the captured graph of its last build, reused across calls."""

    def __init__(self, device: int | None = None):
        torch = _torch()
        if not torch.cuda.is_available():
            raise RuntimeError('the J/K engine needs a CUDA device')
        self.device = torch.cuda.current_device() if device is None else int(device)
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().jk_batch_create(self.device, ctypes.byref(h)), 'jk_batch_create')
        self._h = h
        self._keep = None
        from . import autotune
        table = autotune.load(self.device, 'batch')
        if table:
            autotune.apply(self, table)

    def __del__(self):
        try:
            if self._h is not None:
                _lib.lib().jk_batch_destroy(self._h)
                self._h = None
        except Exception:
            pass

    # ------------------------------------------------------------------
    def _stream(self, stream):
        torch = _torch()
        if stream is None:
            stream = torch.cuda.current_stream(torch.device('cuda', self.device))
        return stream

    def build_async(self, opts, dms, hermi=1, with_j=True, with_k=True, vj=None, vk=None,
                    mixed_threshold=0.0, use_graph=False, stream=None):
        """Enqueue a batched build without synchronising.

        opts: list of built VHFOpt; dms: list of contiguous float64 CUDA
        tensors (n_dm_i, nao_i, nao_i) in each molecule's Cartesian AO basis;
        vj / vk: optional lists of output tensors shaped like dms (allocated
        when None).  Returns (vj, vk) lists (None when not requested)."""
        torch = _torch()
        n = len(opts)
        if n == 0 or len(dms) != n:
            raise ValueError('need one density stack per molecule')
        for o, d in zip(opts, dms):
            if (d.ndim != 3 or d.shape[1] != o.nao or d.shape[2] != o.nao
                    or d.dtype != torch.float64 or not d.is_cuda or not d.is_contiguous()):
                raise ValueError(f'dms must be contiguous float64 CUDA tensors (n_dm, {o.nao}, '
                                 f'{o.nao}); got {tuple(d.shape)} {d.dtype}')
        if with_j and vj is None:
            vj = [torch.empty_like(d) for d in dms]
        if with_k and vk is None:
            vk = [torch.empty_like(d) for d in dms]
        plans = (ctypes.c_void_p * n)(*[o.apply_tol().value for o in opts])
        dmp = (ctypes.c_void_p * n)(*[d.data_ptr() for d in dms])
        ndm = (ctypes.c_int * n)(*[d.shape[0] for d in dms])
        vjp = (ctypes.c_void_p * n)(*[v.data_ptr() for v in vj]) if with_j else None
        vkp = (ctypes.c_void_p * n)(*[v.data_ptr() for v in vk]) if with_k else None
        st = self._stream(stream)
        _lib.check(_lib.lib().jk_batch_build(
            self._h, plans, n, dmp, ndm, int(hermi), int(bool(with_j)), int(bool(with_k)),
            vjp, vkp, float(mixed_threshold), int(bool(use_graph)),
            ctypes.c_void_p(st.cuda_stream)), 'jk_batch_build')
        # the graph of this build reads these buffers: keep them alive
        self._keep = (list(opts), list(dms), vj, vk)
        return vj, vk

    def sync(self, stream=None):
        st = self._stream(stream)
        _lib.check(_lib.lib().jk_batch_sync(self._h, ctypes.c_void_p(st.cuda_stream)),
                   'jk_batch_sync')

    def build(self, opts, dms, hermi=1, with_j=True, with_k=True, vj=None, vk=None,
              mixed_threshold=0.0, use_graph=False, stream=None):
        out = self.build_async(opts, dms, hermi, with_j, with_k, vj, vk, mixed_threshold,
                               use_graph, stream)
        self.sync(stream)
        return out

    # ------------------------------------------------------------------
    def stats(self):
        """{'graph_replayed', 'graph_captured', 'workspace_bytes'} of the last build."""
        r = ctypes.c_int()
        c = ctypes.c_int()
        w = ctypes.c_longlong()
        _lib.check(_lib.lib().jk_batch_stats(self._h, ctypes.byref(r), ctypes.byref(c),
                                             ctypes.byref(w)), 'jk_batch_stats')
        return {'graph_replayed': bool(r.value), 'graph_captured': bool(c.value),
                'workspace_bytes': int(w.value)}

    def class_counts(self, with_f32=False):
        """{(li, lj, lk, ll): (quartets, primitive quartets[, FP32 quartets])}
        of the last build, summed over its molecules."""
        keys = class_keys()
        n = len(keys)
        q = (ctypes.c_ulonglong * n)()
        pq = (ctypes.c_ulonglong * n)()
        q32 = (ctypes.c_ulonglong * n)()
        ncls = ctypes.c_int()
        _lib.check(_lib.lib().jk_batch_counts(self._h, q, pq, q32, n, ctypes.byref(ncls)),
                   'jk_batch_counts')
        return {k: (int(q[i]), int(pq[i])) + ((int(q32[i]),) if with_f32 else ())
                for i, k in enumerate(keys)}

    def set_timing(self, enable=True):
        _lib.check(_lib.lib().jk_batch_set_timing(self._h, int(bool(enable))),
                   'jk_batch_set_timing')

    def last_class_ms(self):
        """({class key: ms of its kernel in the last build}, kernels launched)."""
        keys = class_keys()
        ms = (ctypes.c_float * len(keys))()
        launches = ctypes.c_int()
        _lib.check(_lib.lib().jk_batch_class_ms(self._h, ms, len(keys), ctypes.byref(launches)),
                   'jk_batch_class_ms')
        return {k: float(ms[i]) for i, k in enumerate(keys) if ms[i] > 0}, launches.value

    def set_tuning(self, cls: int, tasks_per_sm: int, blocks_per_sm: int = 0, fp32: int = -1):
        _lib.check(_lib.lib().jk_batch_set_tuning(self._h, int(cls), int(tasks_per_sm),
                                                  int(blocks_per_sm), int(fp32)),
                   'jk_batch_set_tuning')
