"""Build the gpaw_b200 CUDA library (sm_100a) in-tree.

    python -m gpaw_b200.build

Compiles gpaw_b200/csrc/*.cu with nvcc into gpaw_b200/_lib/libgpaw_b200.so.
The library exports only the C ABI declared in include/gpaw_b200.h.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, 'csrc')
OUTDIR = os.path.join(HERE, '_lib')
LIB = os.path.join(OUTDIR, 'libgpaw_b200.so')

ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '-lineinfo', '-std=c++17', '--expt-relaxed-constexpr',
         '-Xcompiler', '-fPIC', '-Xcompiler', '-fvisibility=hidden',
         '-shared']


def nvcc():
    for cand in (os.environ.get('NVCC'), '/usr/local/cuda/bin/nvcc', 'nvcc'):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or
                     not os.path.isabs(cand)):
            return cand
    raise RuntimeError('nvcc not found')


def sources():
    return sorted(glob.glob(os.path.join(CSRC, '*.cu')))


def deps():
    return sources() + sorted(glob.glob(os.path.join(CSRC, '*.cuh'))) + \
        [os.path.join(ROOT, 'include', 'gpaw_b200.h')]


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in deps())


def build(force=False, verbose=False, extra=()):
    if not force and up_to_date():
        return LIB
    os.makedirs(OUTDIR, exist_ok=True)
    cmd = [nvcc(), *ARCH, *FLAGS, *extra, '-I', CSRC,
           '-I', os.path.join(ROOT, 'include'), *sources(), '-o', LIB + '.tmp']
    if verbose:
        print(' '.join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + '.tmp', LIB)
    return LIB


if __name__ == '__main__':
    v = '-v' in sys.argv
    extra = ['-Xptxas', '-v'] if '--ptxas' in sys.argv else []
    print(build(force=True, verbose=v, extra=extra))
