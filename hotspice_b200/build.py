"""Build recipe of libhotspice_sm100.so: nvcc, sm_100a only, in-tree output.

    python -m hotspice_b200.build          # or hotspice_b200.build.build()

Every .cu file compiles to its own object in hotspice_b200/_build/ (in parallel, and only
when the file or a header changed since its object was written); one nvcc call links them.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, 'libhotspice_sm100.so')
OBJ_DIR = os.path.join(HERE, '_build')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-lineinfo', '-O3', '-std=c++17', '-DHS_BUILD', '-Xcompiler', '-fPIC']


def nvcc():
    exe = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
    if not os.path.exists(exe):
        raise RuntimeError('nvcc not found: the CUDA toolkit is required to build hotspice_b200')
    return exe


def sources():
    return sorted(glob.glob(os.path.join(HERE, 'csrc', '*.cu')))


def headers():
    return glob.glob(os.path.join(HERE, 'csrc', '*.cuh')) + glob.glob(os.path.join(HERE, 'csrc', '*.h')) + \
        [os.path.join(os.path.dirname(HERE), 'include', 'hotspice_b200.h')]


def _compile(src, obj, extra, verbose):
    cmd = [nvcc(), *ARCH, *FLAGS, *extra, '-c', '-o', obj + '.tmp', src]
    if verbose:
        print(' '.join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f'nvcc failed on {os.path.basename(src)}:\n{r.stdout}\n{r.stderr}')
    os.replace(obj + '.tmp', obj)
    return obj


def build(verbose: bool = False, force: bool = False, extra=(), out: str | None = None, obj_dir: str | None = None):
    """Compile and link the library; returns its path. ``extra``: more nvcc flags (objects
    built with other flags go to their own ``obj_dir``); ``out``: another output path."""
    out = out or LIB
    obj_dir = obj_dir or OBJ_DIR
    os.makedirs(obj_dir, exist_ok=True)
    srcs = sources()
    newest_header = max(os.path.getmtime(h) for h in headers())
    jobs = []
    objs = []
    for s in srcs:
        o = os.path.join(obj_dir, os.path.basename(s)[:-3] + '.o')
        objs.append(o)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(os.path.getmtime(s), newest_header):
            jobs.append((s, o))
    if not jobs and os.path.exists(out) and os.path.getmtime(out) >= max(os.path.getmtime(o) for o in objs):
        return out
    with cf.ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        list(ex.map(lambda j: _compile(j[0], j[1], list(extra), verbose), jobs))
    cmd = [nvcc(), *ARCH, '-shared', '-o', out + '.tmp', *objs]
    if verbose:
        print(' '.join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f'nvcc link failed:\n{r.stdout}\n{r.stderr}')
    os.replace(out + '.tmp', out)
    return out


if __name__ == '__main__':
    print(build(verbose=True, force='--force' in sys.argv))
