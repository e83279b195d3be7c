"""
Build the in-tree native library ``macromax_b200/libmacromax_b200.so`` for sm_100a with nvcc.

    python -m macromax_b200.build            # rebuild if a source changed
    python -m macromax_b200.build --force    # always rebuild
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, 'csrc')
INCLUDE = os.path.join(ROOT, 'include')
LIB_NAME = 'libmacromax_b200.so'
LIB_PATH = os.path.join(PKG, LIB_NAME)
STAMP = LIB_PATH + '.srchash'

SOURCES = ['mmx_capi.cu']
NVCC_FLAGS = ['-gencode', 'arch=compute_100a,code=sm_100a', '-lineinfo', '-O3', '-std=c++17', '-shared',
              '-Xcompiler', '-fPIC', '-Xcompiler', '-O2']


def _nvcc() -> str:
    for cand in (os.environ.get('NVCC'), shutil.which('nvcc'), '/usr/local/cuda/bin/nvcc'):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError('nvcc not found: set NVCC or put the CUDA toolkit on PATH')


def _source_hash() -> str:
    h = hashlib.sha256()
    for d in (CSRC, INCLUDE):
        for name in sorted(os.listdir(d)):
            if name.endswith(('.cu', '.cuh', '.h')):
                with open(os.path.join(d, name), 'rb') as f:
                    h.update(name.encode())
                    h.update(f.read())
    h.update(' '.join(NVCC_FLAGS).encode())
    return h.hexdigest()


def up_to_date() -> bool:
    if not os.path.exists(LIB_PATH) or not os.path.exists(STAMP):
        return False
    with open(STAMP) as f:
        return f.read().strip() == _source_hash()


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and up_to_date():
        return LIB_PATH
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    tmp = LIB_PATH + '.tmp'
    cmd = [_nvcc(), *NVCC_FLAGS, '-I', INCLUDE, '-o', tmp, *srcs]
    if verbose:
        print(' '.join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, LIB_PATH)
    with open(STAMP, 'w') as f:
        f.write(_source_hash())
    return LIB_PATH


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose=True))
