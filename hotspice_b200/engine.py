"""Batched execution: many Magnets instances advanced by one persistent cluster launch.

The device side is ``hs_engine_run`` (hotspice_b200/csrc/hs_engine.cu): every thread-block
cluster claims instances from a work counter and runs each one's steps with cluster
barriers between the phases of a step, so a whole run of an instance (thousands of steps)
costs one launch instead of two or three kernel launches per step.

Cluster sizes are chosen per instance by :func:`cluster_size_for` (a cost model on the
lattice size and the dipolar window), or measured by :class:`Autotuner`, which times each
candidate on the instance's own shape class and caches the winner.
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .core import Magnets, Scheme

SCHEME_ID = {Scheme.NEEL: 0, Scheme.METROPOLIS: 1, Scheme.WOLFF: 2}
CLUSTER_SIZES = (1, 2, 4, 8, 16)


class HsInstance(ctypes.Structure):
    _fields_ = [('L', _lib.HsLattice), ('P', _lib.HsGridPlan), ('sw', _lib.HsSwitchList),
                ('C', ctypes.c_void_p), ('scratch', ctypes.c_void_p), ('scratch_bytes', ctypes.c_int64),
                ('steps', ctypes.c_int64), ('attempt_freq', ctypes.c_double), ('scheme', ctypes.c_int32),
                ('pad', ctypes.c_int32)]


def _bind():
    lib = _lib.load()
    lib.hs_engine_run.restype = ctypes.c_int
    lib.hs_engine_run.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                                  ctypes.c_void_p]
    lib.hs_engine_max_clusters.restype = ctypes.c_int
    lib.hs_engine_max_clusters.argtypes = [ctypes.c_int32]
    sizes = (ctypes.c_int32 * 6)()
    lib.hs_struct_sizes(sizes, 6)
    if sizes[5] != ctypes.sizeof(HsInstance):
        raise RuntimeError(f'HsInstance ABI mismatch: {sizes[5]} != {ctypes.sizeof(HsInstance)}')
    return lib


def cluster_size_for(mm: Magnets) -> int:
    """Cost model: enough CTAs that one step's scan / update work (cells times window)
    is spread thin, but no more (cluster barriers cost more with more CTAs)."""
    n = mm.nx * mm.ny
    d = mm._dipolar()
    win = 0
    if d is not None:
        ks = d.kernel_set
        win = (2 * ks.wx + 1) * (2 * ks.wy + 1)
    if mm.params.UPDATE_SCHEME == Scheme.NEEL:
        work = n + win
    elif mm.params.UPDATE_SCHEME == Scheme.WOLFF:
        return 1
    else:
        work = win * 8
    if work <= 16384:
        return 1
    if work <= 65536:
        return 2
    if work <= 262144:
        return 4
    if work <= 1048576:
        return 8
    return 16


@dataclass
class _Prepared:
    inst: torch.Tensor
    n: int
    cs: int
    keep: list


class BatchEngine:
    """Advance several Magnets at once: ``run(steps)`` (fixed step budgets) or
    ``progress(t_max, MCsteps_max)`` (the reference's stop rule, per instance)."""

    def __init__(self, magnets, cluster_size: int | None = None, device=None):
        self.magnets = list(magnets)
        if not self.magnets:
            raise ValueError('BatchEngine needs at least one Magnets instance')
        self.device = torch.device(device) if device is not None else self.magnets[0].device
        for mm in self.magnets:
            if mm.device != self.device:
                raise ValueError('all instances of a BatchEngine must live on the same device')
        self.cluster_size = cluster_size
        self.lib = _bind()
        self._work = torch.zeros(1, device=self.device, dtype=torch.int32)
        self._max_clusters = {}

    def _max(self, cs):
        if cs not in self._max_clusters:
            n = self.lib.hs_engine_max_clusters(cs)
            if n < 0:
                raise RuntimeError(_lib.last_error())
            self._max_clusters[cs] = max(1, n)
        return self._max_clusters[cs]

    def _describe(self, mm: Magnets, steps: int, kw) -> tuple[HsInstance, list]:
        kind, L, s, extra, buf = mm._step_args(kw)
        I = HsInstance()
        I.L = L
        I.sw = s
        I.C = mm._counters.data_ptr()
        I.scratch = buf.data_ptr()
        I.scratch_bytes = buf.numel()
        I.steps = int(steps)
        I.scheme = SCHEME_ID[mm.params.UPDATE_SCHEME]
        if kind == 'metro':
            I.P = extra
            I.attempt_freq = extra.attempt_freq
        elif kind == 'neel':
            I.attempt_freq = extra
        else:
            I.attempt_freq = 1e10
        return I, [buf, s]

    def _prepare(self, steps, kws):
        groups = {}
        keep = []
        for mm, st, kw in zip(self.magnets, steps, kws):
            if mm._T_zero:
                raise RuntimeError('an instance has T=0 somewhere in its domain')
            cs = self.cluster_size or getattr(mm, '_cluster_size', None) or cluster_size_for(mm)
            I, k = self._describe(mm, st, kw)
            keep += k
            groups.setdefault(cs, []).append(I)
        out = []
        for cs, lst in sorted(groups.items()):
            arr = (HsInstance * len(lst))(*lst)
            raw = np.frombuffer(bytes(arr), dtype=np.uint8)
            t = torch.from_numpy(raw.copy()).to(self.device)
            out.append(_Prepared(t, len(lst), cs, keep))
        return out

    def launch(self, prepared, stream=None):
        st = stream if stream is not None else torch.cuda.current_stream(self.device).cuda_stream
        for p in prepared:
            n_clusters = min(p.n, self._max(p.cs))
            work = self._work
            _lib.check(self.lib.hs_engine_run(p.inst.data_ptr(), p.n, p.cs, n_clusters, work.data_ptr(), st),
                       'hs_engine_run')

    def run(self, steps, **kwargs):
        """Enqueue ``steps`` (an int or one int per instance) update steps of every instance
        without the stop rule; asynchronous."""
        steps = [int(steps)] * len(self.magnets) if np.isscalar(steps) else [int(s) for s in steps]
        kws = [dict(kwargs) for _ in self.magnets]
        for mm, kw in zip(self.magnets, kws):
            mm._set_control(progress=0, done=0, t_max=float(kw.pop('t_max', math.inf)))
        prepared = self._prepare(steps, kws)
        self.launch(prepared)
        return prepared

    def progress(self, t_max=1.0, MCsteps_max=4.0, **kwargs):
        """The reference's progress() for every instance at once; returns [(dt, dMCsteps)]."""
        starts = []
        for mm in self.magnets:
            c = mm._read_counters()
            t0, mc0 = float(c['t']), float(c['attempted']) / mm.n
            mm._write_counters(t0=t0, mc0=mc0, t_max=float(t_max), mc_max=float(MCsteps_max), progress=1, done=0)
            starts.append((t0, mc0))
        prepared = self._prepare([0] * len(self.magnets), [dict(kwargs) for _ in self.magnets])
        self.launch(prepared)
        out = []
        for mm, (t0, mc0) in zip(self.magnets, starts):
            c = mm._read_counters()
            st = int(c['status'])
            if st:
                raise RuntimeError(f'device step reported status {st} (HS_ST_* bits)')
            mm._write_counters(progress=0, done=0)
            out.append((float(c['t']) - t0, float(c['attempted']) / mm.n - mc0))
        return out


class Autotuner:
    """Measures each cluster size on an instance (a copy of its state is restored afterwards)
    and caches the fastest per shape class (lattice type, nx, ny, scheme, window)."""

    def __init__(self):
        self.cache = {}

    @staticmethod
    def key(mm: Magnets):
        d = mm._dipolar()
        win = (d.kernel_set.wx, d.kernel_set.wy) if d is not None else (0, 0)
        return (type(mm).__name__, mm.nx, mm.ny, mm.params.UPDATE_SCHEME, mm.params.MULTISAMPLING_SCHEME, win)

    def tune(self, mm: Magnets, steps=200, candidates=CLUSTER_SIZES, **kw) -> int:
        k = self.key(mm)
        if k in self.cache:
            mm._cluster_size = self.cache[k]
            return self.cache[k]
        snap = mm._snapshot()
        best, best_t = None, math.inf
        for cs in candidates:
            eng = BatchEngine([mm], cluster_size=cs)
            eng.run(max(steps // 10, 5), **kw)  # warm-up
            torch.cuda.synchronize(mm.device)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            eng.run(steps, **kw)
            e1.record()
            torch.cuda.synchronize(mm.device)
            t = e0.elapsed_time(e1)
            mm._restore(snap)
            if t < best_t:
                best, best_t = cs, t
        self.cache[k] = best
        mm._cluster_size = best
        return best
