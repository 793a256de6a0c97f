"""Build libjk_b200.so (sm_100a) in-tree.

    python -m electrolites_b200.build [-j N] [--lmax L]

Steps: generate the Rys tables and the per-class kernel sources
(codegen/rys_table.py, codegen/gen_classes.py) into csrc/generated/, compile
each translation unit with nvcc for sm_100a in parallel, link the shared
library next to this file.  Objects are cached by a hash of their inputs in
csrc/_build/.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
GEN = os.path.join(CSRC, 'generated')
OBJ = os.path.join(CSRC, '_build')
LIB = os.path.join(HERE, 'libjk_b200.so')
ROOT = os.path.dirname(HERE)

NVCC_FLAGS = ['-gencode', 'arch=compute_100a,code=sm_100a', '-lineinfo', '-O3',
              '-std=c++17', '-Xcompiler', '-fPIC', '-Xcompiler', '-O2',
              '--expt-relaxed-constexpr', '-Xptxas', '-v']


def nvcc() -> str:
    p = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
    if not os.path.exists(p):
        raise RuntimeError('nvcc not found')
    return p


def generate():
    sys.path.insert(0, ROOT)
    from electrolites_b200.codegen import gen_classes, rys_table
    dims = os.path.join(GEN, 'rys_table_dims.inc')
    data = os.path.join(GEN, 'rys_table_data.inc')
    stamp = os.path.join(GEN, '.rys_stamp')
    src_hash = hashlib.sha1(open(rys_table.__file__, 'rb').read()).hexdigest()
    if not (os.path.exists(dims) and os.path.exists(data) and os.path.exists(stamp)
            and open(stamp).read() == src_hash):
        rys_table.write_include(GEN)
        with open(stamp, 'w') as f:
            f.write(src_hash)
    return gen_classes.write_all(GEN)


def _deps_hash(src: str) -> str:
    h = hashlib.sha1()
    h.update(' '.join(NVCC_FLAGS).encode())
    for p in [src] + sorted(
            os.path.join(CSRC, f) for f in os.listdir(CSRC)
            if f.endswith(('.cuh', '.h'))) + [
            os.path.join(GEN, 'rys_table_dims.inc'),
            os.path.join(ROOT, 'include', 'jk_b200.h')]:
        h.update(open(p, 'rb').read())
    if src.endswith('jk_api.cu'):
        for f in ('class_table.inc', 'rys_table_data.inc'):
            h.update(open(os.path.join(GEN, f), 'rb').read())
    return h.hexdigest()[:16]


def _compile(src: str) -> tuple[str, str]:
    base = os.path.splitext(os.path.basename(src))[0]
    obj = os.path.join(OBJ, f'{base}.{_deps_hash(src)}.o')
    if os.path.exists(obj):
        return obj, ''
    cmd = [nvcc()] + NVCC_FLAGS + ['-I', CSRC, '-c', src, '-o', obj + '.tmp']
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f'nvcc failed for {src}:\n{r.stderr[-6000:]}')
    os.replace(obj + '.tmp', obj)
    with open(os.path.join(OBJ, f'{base}.ptxas.txt'), 'w') as f:
        f.write(r.stderr)
    return obj, r.stderr


def build(jobs: int = 0, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    units = generate()
    units = [os.path.join(CSRC, 'jk_api.cu')] + units
    jobs = jobs or max(1, os.cpu_count() or 1)
    objs = []
    with cf.ThreadPoolExecutor(jobs) as ex:
        for obj, log in ex.map(_compile, units):
            objs.append(obj)
            if verbose and log:
                print(log)
    tmp = LIB + '.tmp'
    cmd = [nvcc(), '-shared', '-gencode', 'arch=compute_100a,code=sm_100a',
           '-o', tmp] + objs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f'link failed:\n{r.stderr[-4000:]}')
    os.replace(tmp, LIB)
    keep = {os.path.basename(o) for o in objs}
    for f in os.listdir(OBJ):
        if f.endswith('.o') and f not in keep:
            os.unlink(os.path.join(OBJ, f))
    return LIB


if __name__ == '__main__':
    ap = argparse.ArgumentParser()
    ap.add_argument('-j', type=int, default=0)
    ap.add_argument('-v', action='store_true')
    a = ap.parse_args()
    print(build(a.j, a.v))
