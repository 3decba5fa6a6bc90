"""Build recipe of libhotspice_sm100.so: nvcc, sm_100a only, in-tree output.

    python -m hotspice_b200.build          # or hotspice_b200.build.build()
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, 'libhotspice_sm100.so')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']


def nvcc():
    exe = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
    if not os.path.exists(exe):
        raise RuntimeError('nvcc not found: the CUDA toolkit is required to build hotspice_b200')
    return exe


def sources():
    return sorted(glob.glob(os.path.join(HERE, 'csrc', '*.cu')))


def build(verbose: bool = False, force: bool = False, extra=()):
    srcs = sources()
    deps = srcs + glob.glob(os.path.join(HERE, 'csrc', '*.cuh')) + glob.glob(os.path.join(HERE, 'csrc', '*.h')) + \
        [os.path.join(os.path.dirname(HERE), 'include', 'hotspice_b200.h')]
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(d) for d in deps):
        return LIB
    cmd = [nvcc(), *ARCH, '-lineinfo', '-O3', '-std=c++17', '-DHS_BUILD',
           '-Xcompiler', '-fPIC', '-shared', '-o', LIB + '.tmp', *srcs, *extra]
    if verbose:
        print(' '.join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f'nvcc failed:\n{r.stdout}\n{r.stderr}')
    if verbose and r.stderr:
        print(r.stderr)
    os.replace(LIB + '.tmp', LIB)
    return LIB


if __name__ == '__main__':
    print(build(verbose=True, force='--force' in sys.argv))
