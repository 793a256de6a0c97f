"""ctypes binding of libjk_b200.so (include/jk_b200.h).

The library is built in-tree by `python -m electrolites_b200.build`.  There
is no fallback: if it is missing or cannot be loaded, every entry point of
the package raises.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'libjk_b200.so')

JK_ERRORS = {1: 'invalid argument', 2: 'unsupported shell', 3: 'CUDA error',
             4: 'out of device memory', 5: 'density out of the plan range',
             6: 'kernel error flag', 7: 'beyond the allocation-free scratch'}

EXPORTS = ['jk_plan_create', 'jk_plan_destroy', 'jk_plan_info', 'jk_build',
           'jk_build_host', 'jk_sync', 'jk_last_counts', 'jk_class_info',
           'jk_set_timing', 'jk_last_class_ms', 'jk_fp64_peak', 'jk_build_noalloc',
           'jk_plan_q_cond', 'jk_build_rs', 'jk_build_op', 'jk_plan_memory', 'jk_plan_set_shard',
           'jk_plan_set_tol', 'jk_plan_set_jengine', 'jk_plan_set_tuning',
           'jk_batch_create', 'jk_batch_destroy', 'jk_batch_build', 'jk_batch_sync',
           'jk_batch_counts', 'jk_batch_set_timing', 'jk_batch_class_ms',
           'jk_batch_set_tuning', 'jk_batch_stats', 'jk_last_error', 'jk_grad',
           'jk_plan_set_jmd']

_lib = None


class JKError(RuntimeError):
    def __init__(self, code, where):
        msg = lib().jk_last_error().decode(errors='replace')
        super().__init__(f'{where}: {JK_ERRORS.get(code, code)} ({code}): {msg}')
        self.code = code


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f'{LIB_PATH} is not built: run '
                           '`python -m electrolites_b200.build`')
    L = ctypes.CDLL(LIB_PATH)
    vp, ip, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.c_void_p
    c_int, c_double = ctypes.c_int, ctypes.c_double
    L.jk_plan_create.argtypes = [vp, c_int, vp, c_int, vp, vp, c_double, c_int,
                                 ctypes.POINTER(vp)]
    L.jk_plan_destroy.argtypes = [vp]
    L.jk_plan_info.argtypes = [vp, ip, ctypes.POINTER(ctypes.c_longlong)]
    L.jk_build.argtypes = [vp, dp, c_int, c_int, c_int, c_int, dp, dp, c_double, vp]
    L.jk_build_host.argtypes = [vp, dp, c_int, c_int, c_int, c_int, dp, dp, c_double, vp]
    L.jk_build_noalloc.argtypes = [vp, dp, c_int, c_int, c_int, c_int, dp, dp, c_double, vp]
    L.jk_build_rs.argtypes = [vp, dp, c_int, c_int, c_int, c_int, dp, dp, c_double, c_double, vp]
    L.jk_build_op.argtypes = [vp, dp, c_int, c_int, c_int, c_int, dp, dp, c_double, c_int, vp, vp,
                              vp]
    L.jk_sync.argtypes = [vp, vp]
    L.jk_grad.argtypes = [vp, dp, c_int, c_double, c_double, c_double, dp, vp]
    L.jk_last_counts.argtypes = [vp, ctypes.POINTER(ctypes.c_ulonglong),
                                 ctypes.POINTER(ctypes.c_ulonglong),
                                 ctypes.POINTER(ctypes.c_ulonglong), c_int, ip]
    L.jk_class_info.argtypes = [c_int, ip, ip, ip, ip, ip]
    L.jk_plan_q_cond.argtypes = [vp, ctypes.POINTER(ctypes.c_float), c_int]
    L.jk_set_timing.argtypes = [vp, c_int]
    L.jk_last_class_ms.argtypes = [vp, ctypes.POINTER(ctypes.c_float), c_int, ip]
    L.jk_fp64_peak.argtypes = [c_int, ctypes.POINTER(ctypes.c_double)]
    llp = ctypes.POINTER(ctypes.c_longlong)
    ullp = ctypes.POINTER(ctypes.c_ulonglong)
    L.jk_plan_memory.argtypes = [vp, llp, llp]
    L.jk_plan_set_shard.argtypes = [vp, c_int, c_int]
    L.jk_plan_set_tol.argtypes = [vp, c_double]
    L.jk_plan_set_jengine.argtypes = [vp, c_int]
    L.jk_plan_set_tuning.argtypes = [vp, c_int, c_int, c_int, c_int]
    L.jk_plan_set_jmd.argtypes = [vp, c_int, c_int]
    L.jk_batch_create.argtypes = [c_int, ctypes.POINTER(vp)]
    L.jk_batch_destroy.argtypes = [vp]
    L.jk_batch_build.argtypes = [vp, vp, c_int, vp, vp, c_int, c_int, c_int, vp, vp, c_double,
                                 c_int, vp]
    L.jk_batch_sync.argtypes = [vp, vp]
    L.jk_batch_counts.argtypes = [vp, ullp, ullp, ullp, c_int, ip]
    L.jk_batch_set_timing.argtypes = [vp, c_int]
    L.jk_batch_class_ms.argtypes = [vp, ctypes.POINTER(ctypes.c_float), c_int, ip]
    L.jk_batch_set_tuning.argtypes = [vp, c_int, c_int, c_int, c_int]
    L.jk_batch_stats.argtypes = [vp, ip, ip, llp]
    L.jk_last_error.restype = ctypes.c_char_p
    for name in EXPORTS:
        if name != 'jk_last_error':
            getattr(L, name).restype = c_int
    _lib = L
    return L


def check(code, where):
    if code != 0:
        raise JKError(code, where)
