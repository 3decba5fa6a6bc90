"""Batched execution: many Magnets instances advanced by one persistent cluster launch.

The device side is ``hs_engine_run`` (hotspice_b200/csrc/hs_engine.cu): every thread-block
cluster claims instances from a work counter and runs each one's steps with cluster
barriers between the phases of a step, so a whole run of an instance (thousands of steps)
costs one launch instead of two or three kernel launches per step.

Cluster sizes are chosen per instance by :func:`cluster_size_for` (a cost model on the
lattice size and the dipolar window), or measured by :class:`Autotuner`, which times each
candidate on the instance's own shape class and caches the winner. A batch runs as one launch
whose longest runs take whole clusters and whose others run on single CTAs of the clusters that
split (:func:`plan_split` on the model, or :meth:`BatchEngine.tune_split` on the device).
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
                ('flags', ctypes.c_int32)]


def _bind():
    lib = _lib.load()
    lib.hs_engine_run_ws.restype = ctypes.c_int
    lib.hs_engine_run_ws.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                                     ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p]
    lib.hs_engine_max_clusters.restype = ctypes.c_int
    lib.hs_engine_max_clusters.argtypes = [ctypes.c_int32]
    sizes = (ctypes.c_int32 * 6)()
    lib.hs_struct_sizes(sizes, 6)
    if sizes[5] != ctypes.sizeof(HsInstance):
        raise RuntimeError(f'HsInstance ABI mismatch: {sizes[5]} != {ctypes.sizeof(HsInstance)}')
    return lib


def step_model(mm: Magnets) -> tuple[float, float, float]:
    """Device time of one step as (fixed us, cell-dependent us on one CTA, exponent alpha): on a
    cluster of cs CTAs a step takes fixed + part / cs**alpha. Calibrated on B200 with single
    instances of the bench lattices (n = 32..512, cluster sizes 1, 4, 16): the cell-dependent
    part grows like c N^beta with the lattice's occupancy class (dense / half / sparse, which
    also carries the perpendicular channel of the in-plane lattices), Néel scans spread over the
    cluster like cs^0.62 and Metropolis steps like cs^0.5; a Wolff step grows its cluster on one
    CTA and costs 10-17 us above the critical temperature. Inside a full batch the model ranks
    runs less well (it underestimates how much two CTAs speed up a large Néel scan), so a
    batch's launch plan is best measured (:meth:`BatchEngine.tune_split`)."""
    n = mm.nx * mm.ny
    f = mm.n / max(n, 1)
    cls = 0 if f >= 0.75 else (1 if f >= 0.45 else 2)
    sch = mm.params.UPDATE_SCHEME
    if sch == Scheme.NEEL:
        c, beta = ((0.0116, 0.786), (0.0198, 0.716), (0.0431, 0.646))[cls]
        return 9.0, c * n ** beta, 0.62
    if sch == Scheme.WOLFF:
        return 11.0 + 6e-6 * n, 0.0, 0.0
    c, beta = ((0.0037, 0.70), (0.0068, 0.70), (0.0061, 0.73))[cls]
    return 5.0, c * n ** beta, 0.5


def model_time(m, cs):
    """Step time (us) of a step model (fixed us, cell-dependent us, alpha) on ``cs`` CTAs."""
    s0, p, alpha = m
    return s0 + (p / cs ** alpha if alpha > 0 else p) + 0.1 * (cs - 1)


def step_time(mm: Magnets, cs: int = 1) -> float:
    """Modelled device time (us) of one step of ``mm`` on a cluster of ``cs`` CTAs."""
    return model_time(step_model(mm), cs)


def step_cost(mm: Magnets) -> float:
    """Cost of one update step in SM-microseconds (the model on one CTA)."""
    return step_time(mm, 1)


def cluster_size_for(mm: Magnets) -> int:
    """Cluster size for an instance run alone: double the CTAs while that cuts the modelled
    step time by at least 25%."""
    cs = 1
    while cs < 16 and step_time(mm, 2 * cs) < 0.75 * step_time(mm, cs):
        cs *= 2
    return cs


def lpt_makespan(durations, n_workers):
    """Makespan of longest-processing-time-first list scheduling of ``durations`` on
    ``n_workers`` identical workers (what the engine's work counter does with instances
    sorted longest first)."""
    import heapq
    if n_workers <= 0:
        return math.inf
    heap = [0.0] * min(n_workers, max(1, len(durations)))
    for d in sorted(durations, reverse=True):
        t = heapq.heappop(heap)
        heapq.heappush(heap, t + d)
    return max(heap)


def plan_uniform_size(models, steps, n_sm, sizes=CLUSTER_SIZES, workers=None):
    """One cluster size for a whole launch: the size whose longest-first schedule of the
    modelled run times over the clusters that fit (``workers[cs]``, the resident clusters of
    that size, else SM count / size) finishes first. One size per launch keeps clusters of
    different shapes from fragmenting the GPCs."""
    t = model_time
    best, best_t = 1, math.inf
    for cs in sizes:
        nw = workers[cs] if workers else n_sm // cs
        mk = lpt_makespan([st * t(m, cs) for m, st in zip(models, steps)], nw)
        if mk < best_t * 0.97:
            best, best_t = cs, mk
    return best


def split_makespan(cluster_runs, cta_runs, n_clusters, cs):
    """Makespan of a split launch (HS_INST_ONE_CTA): ``n_clusters`` clusters of ``cs`` CTAs
    take the ``cluster_runs`` longest first; each cluster that finds no more of them splits,
    and its CTAs take the ``cta_runs`` (run times on one CTA) longest first."""
    import heapq
    heap = [0.0] * max(1, n_clusters)
    for d in sorted(cluster_runs, reverse=True):
        heapq.heappush(heap, heapq.heappop(heap) + d)
    ctas = [t for t in heap for _ in range(cs)]
    heapq.heapify(ctas)
    for d in sorted(cta_runs, reverse=True):
        heapq.heappush(ctas, heapq.heappop(ctas) + d)
    return max(ctas)


def plan_split(models, steps, workers, sizes=CLUSTER_SIZES):
    """Cluster size and per-instance mode of one launch: the k longest runs (by their time on
    one CTA) use whole clusters of ``cs`` CTAs, the others one CTA each (the engine's split
    mode). Every size and a grid of k (k = n: one size for all) are simulated with
    :func:`split_makespan` over the modelled run times; ``workers[cs]`` is the number of
    resident clusters of each size. Returns (cs, one_cta flags, modelled makespan in us)."""
    t = model_time
    n = len(models)
    d1 = [st * t(m, 1) for m, st in zip(models, steps)]
    order = sorted(range(n), key=lambda i: (-d1[i], i))
    best = (lpt_makespan(d1, workers[1]), 1, n)
    ks = sorted(set(range(0, n + 1, max(1, n // 64))) | {n})
    for cs in sizes:
        if cs == 1:
            continue
        dc = [st * t(m, cs) for m, st in zip(models, steps)]
        for k in ks:
            mk = split_makespan([dc[i] for i in order[:k]], [d1[i] for i in order[k:]], workers[cs], cs)
            if mk < best[0] * 0.99:
                best = (mk, cs, k)
    mk, cs, k = best
    flags = [False] * n
    if cs > 1:
        for i in order[k:]:
            flags[i] = True
    return cs, flags, mk


def plan_sizes(models, steps, n_sm, max_cs=16):
    """Cluster sizes for a batch: start every instance on one CTA; an instance whose run is
    longer than the even share of the GPU (total SM time / SM count) gets twice the CTAs
    while that shortens it by at least 20%, until no run exceeds the share (or max_cs).
    ``models``: (fixed us, cell-dependent us, alpha) per instance, as step_model gives."""
    t = model_time
    cs = [1] * len(models)
    for _ in range(5):
        share = sum(st * t(m, c) * c for m, st, c in zip(models, steps, cs)) / n_sm
        changed = False
        for i, (m, st) in enumerate(zip(models, steps)):
            while cs[i] < max_cs and m[2] > 0 and st * t(m, cs[i]) > share and t(m, 2 * cs[i]) < 0.8 * t(m, cs[i]):
                cs[i] *= 2
                changed = True
        if not changed:
            break
    return cs


@dataclass
class _Prepared:
    inst: torch.Tensor
    n: int
    cs: int
    keep: list
    ws: int = 0         # dynamic shared workspace per CTA (bytes)
    order: list = None  # index into the engine's instance list of each launch slot
    ns: torch.Tensor = None   # device time (ns) of each launch slot, written by the launch
    one_cta: int = 0    # instances that run on one CTA of a split cluster (HS_INST_ONE_CTA)


def poisson_workspace(I: HsInstance) -> int:
    """Shared workspace bytes that hold a Poisson-disc Metropolis instance's sampler arrays
    (24 bytes per background-grid cell + 64; the grid has cells of side (r+1)/sqrt(2) over the
    lattice, hotspice/poisson.py:78-83), 0 for every other instance or when they exceed the
    largest workspace (the sampler then works in the instance's scratch)."""
    if I.scheme != SCHEME_ID[Scheme.METROPOLIS] or I.P.sample_scheme != _lib.HS_SAMPLE_POISSON:
        return 0
    cs = (I.P.r_cells + 1.0) / math.sqrt(2.0)
    need = 24 * math.ceil(I.L.nx / cs) * math.ceil(I.L.ny / cs) + 64
    return need if need <= _lib.HS_ENGINE_WS_MAX else 0


class CapturedRun:
    """A CUDA graph holding one engine launch (see :meth:`BatchEngine.capture`); it keeps the
    instance descriptors it points to alive."""

    def __init__(self, graph, prepared, engine):
        self.graph, self.prepared, self.engine = graph, prepared, engine

    def replay(self):
        self.graph.replay()


SEGMENT_DTYPE = np.dtype([('staged', '<i8'), ('device', '<u8'), ('bytes', '<i8')])   # HsSegment


def segment_table(layout, ptrs, max_bytes=None) -> np.ndarray:
    """HsSegment rows for a packed layout [(instance, field, staged offset, bytes)] and the
    arrays' device addresses: every array split into pieces of at most ``max_bytes``
    (HS_SEGMENT_MAX), each piece starting at the same offset into both sides."""
    max_bytes = _lib.HS_SEGMENT_MAX if max_bytes is None else int(max_bytes)
    rows = []
    for (_, _, off, nb), p in zip(layout, ptrs):
        for k in range(0, nb, max_bytes):
            rows.append((off + k, p + k, min(max_bytes, nb - k)))
    return np.array(rows, dtype=SEGMENT_DTYPE)


class BatchEngine:
    """Advance several Magnets at once: ``run(steps)`` (fixed step budgets) or
    ``progress(t_max, MCsteps_max)`` (the reference's stop rule, per instance)."""

    def __init__(self, magnets, cluster_size: int | None = None, device=None, throughput: bool | None = None):
        """``throughput``: plan one cluster size for the launch from the modelled run times
        (:func:`plan_uniform_size`); default on when there is more than one instance, otherwise
        the instance's own size (:func:`cluster_size_for` or its autotuned choice)."""
        self.magnets = list(magnets)
        if not self.magnets:
            raise ValueError('BatchEngine needs at least one Magnets instance')
        self.device = torch.device(device) if device is not None else self.magnets[0].device
        for mm in self.magnets:
            if mm.device != self.device:
                raise ValueError('all instances of a BatchEngine must live on the same device')
        self.cluster_size = cluster_size
        if throughput is None:
            throughput = len(self.magnets) > 1
        self.throughput = throughput
        self._cache = None
        self._streams = []
        self.lib = _bind()
        # one work counter per cluster-size group, never reallocated (launches in flight use them)
        self._work = torch.zeros(len(CLUSTER_SIZES), device=self.device, dtype=torch.int32)
        self._max_clusters = {}
        self._desc = {}     # id(mm) -> (version, kw key, HsInstance, buffers it points into)
        self._tuned = None  # (step budgets, sizes, one-CTA flags) measured best by tune_split

    def set_magnets(self, magnets):
        """Replace the instance list (a serving loop changes it between launches); descriptors
        of instances that stay are reused."""
        self.magnets = list(magnets)
        if not self.magnets:
            raise ValueError('BatchEngine needs at least one Magnets instance')
        live = {id(mm) for mm in self.magnets}
        self._desc = {k: v for k, v in self._desc.items() if k in live}
        self._cache = None
        self._tuned = None

    def _max(self, cs):
        if cs not in self._max_clusters:
            n = self.lib.hs_engine_max_clusters(cs)
            if n < 0:
                raise RuntimeError(_lib.last_error())
            self._max_clusters[cs] = max(1, n)
        return self._max_clusters[cs]

    def _describe_cached(self, mm: Magnets, steps: int, kw) -> tuple[HsInstance, list]:
        key = (mm._version, tuple(sorted((k, float(v)) for k, v in kw.items())))
        hit = self._desc.get(id(mm))
        if hit is None or hit[0] is not mm or hit[1] != key:
            I, keep = self._describe(mm, steps, kw)
            self._desc[id(mm)] = hit = (mm, key, I, keep)
        I = HsInstance.from_buffer_copy(hit[2])
        I.steps = int(steps)
        return I, hit[3]

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

    def _throughput_sizes(self, steps):
        """Cluster size and per-instance CTA mode for throughput mode: one launch whose longest
        runs use whole clusters and whose others run on one CTA each (:func:`plan_split` over
        the modelled step times), or the plan :meth:`tune_split` measured for these budgets."""
        if self._tuned is not None and self._tuned[0] == tuple(steps):
            return list(self._tuned[1]), list(self._tuned[2])
        cs, flags, _ = plan_split([step_model(mm) for mm in self.magnets], [max(1, st) for st in steps],
                                  {c: self._max(c) for c in CLUSTER_SIZES})
        return [cs] * len(self.magnets), flags

    def _prepare(self, steps, kws, sizes=None, costs=None, one_cta=None):
        groups = {}
        keep = []
        tsizes = None
        if one_cta is None and self.throughput and not self.cluster_size and not sizes:
            tsizes, one_cta = self._throughput_sizes(steps)
        for j, (mm, st, kw) in enumerate(zip(self.magnets, steps, kws)):
            if mm._T_zero:
                raise RuntimeError('an instance has T=0 somewhere in its domain')
            cs = (sizes[j] if sizes else None) or self.cluster_size or (tsizes[j] if tsizes else None) \
                or getattr(mm, '_cluster_size', None) or cluster_size_for(mm)
            if cs not in CLUSTER_SIZES:
                raise ValueError(f'cluster size {cs} not in {CLUSTER_SIZES}')
            I, k = self._describe_cached(mm, st, kw)
            keep += k
            alone = bool(one_cta and one_cta[j])
            I.flags = _lib.HS_INST_ONE_CTA if alone else 0
            cost = costs[j] if costs is not None else st * step_time(mm, 1 if alone else cs)
            groups.setdefault(cs, []).append((alone, cost, j, I))
        out = []
        # the workspace only for groups with Poisson-disc instances: it takes L1 from the rest
        # largest clusters first (launched first, so the longest runs start first), and inside a
        # group the longest runs first on the work counter (longest-processing-time order),
        # the instances that run on one CTA after all that use whole clusters
        for cs, lst in sorted(groups.items(), reverse=True):
            lst = sorted(lst, key=lambda e: (e[0], -e[1], e[2]))
            order = [j for _, _, j, _ in lst]
            n_one = sum(1 for e in lst if e[0])
            lst = [I for _, _, _, I in lst]
            arr = (HsInstance * len(lst))(*lst)
            raw = np.frombuffer(bytes(arr), dtype=np.uint8)
            # pinned staging + asynchronous copy on the current stream: no host synchronisation
            t = torch.from_numpy(raw.copy()).pin_memory().to(self.device, non_blocking=True)
            ws = max(poisson_workspace(I) for I in lst)
            out.append(_Prepared(t, len(lst), cs, keep, (ws + 1023) // 1024 * 1024, order,
                                 torch.zeros(len(lst), dtype=torch.int64, device=self.device), n_one))
        return out

    def launch(self, prepared, stream=None):
        """One engine launch per cluster-size group; several groups run concurrently on side
        streams that join the caller's stream again."""
        main = torch.cuda.current_stream(self.device) if stream is None else stream
        if len(prepared) == 1:
            self._launch_one(prepared[0], 0, main.cuda_stream)
            return
        if len(self._streams) < len(prepared):
            self._streams += [torch.cuda.Stream(self.device) for _ in range(len(prepared) - len(self._streams))]
        for g, p in enumerate(prepared):
            s = self._streams[g]
            s.wait_stream(main)
            self._launch_one(p, g, s.cuda_stream)
        for g in range(len(prepared)):
            main.wait_stream(self._streams[g])

    def _launch_one(self, p, g, st):
        n_clusters = min(p.n, self._max(p.cs))
        _lib.check(self.lib.hs_engine_run_ws(p.inst.data_ptr(), p.n, p.cs, n_clusters, self._work[g:].data_ptr(),
                                             p.ws, p.ns.data_ptr(), st), 'hs_engine_run_ws')

    def tune_split(self, steps, reps: int = 2, sizes=(2, 4), ks=None, **kwargs):
        """Measure split launches of throughput mode on the device and keep the fastest plan for
        these step budgets (``run`` and ``capture`` use it until the instance list changes).
        One launch with every instance on one CTA measures each instance's run time (the
        engine's per-instance device time); the instances are ranked by it, and for each cluster
        size in ``sizes`` and each k in ``ks`` the k longest run on whole clusters and the rest
        on one CTA each, timed over ``reps`` launches after one warm-up launch. The instances'
        state (spins, moments, energies, counters) is saved on the device first and restored
        afterwards, so tuning leaves the simulations where they were. Returns (cluster size, k,
        ms per launch) of the plan kept."""
        if not self.throughput or self.cluster_size:
            raise ValueError('tune_split plans throughput-mode launches: create the BatchEngine with '
                             'throughput=True and no fixed cluster_size')
        n = len(self.magnets)
        steps_l = [int(steps)] * n if np.isscalar(steps) else [int(x) for x in steps]
        if ks is None:
            ks = [k for k in (4, 8, 12, 16, 24, 32, 40, 48, 64, 96, 128, 192) if k < n] + [n]
        stream = torch.cuda.current_stream(self.device)
        stage, total = self._gather(self.STATE_FIELDS, stream.cuda_stream)
        saved = stage[:total].clone()

        def timed(cs, flags):
            self._tuned = (tuple(steps_l), [cs] * n, [bool(f) for f in flags])
            self._cache = None
            prep = self.run(steps_l, **kwargs)
            best = math.inf
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                prep = self.run(steps_l, **kwargs)
                e1.record(stream)
                e1.synchronize()
                best = min(best, e0.elapsed_time(e1))
            return best, prep

        reps = max(1, int(reps))
        try:
            t_one, prep = timed(max(sizes), [True] * n)   # every instance on one CTA
            d1 = np.zeros(n)
            for p in prep:
                ns = p.ns.cpu().numpy()
                for slot, j in enumerate(p.order):
                    d1[j] = ns[slot]
            order = np.argsort(-d1, kind='stable')
            best = (t_one, max(sizes), 0)
            for cs in sizes:
                for k in ks:
                    flags = np.ones(n, dtype=bool)
                    flags[order[:k]] = False
                    t, _ = timed(cs, flags)
                    if t < best[0]:
                        best = (t, cs, k)
            t, cs, k = best
            flags = np.ones(n, dtype=bool)
            flags[order[:k]] = False
            self._tuned = (tuple(steps_l), [cs] * n, [bool(f) for f in flags])
        except BaseException:
            self._tuned = None
            raise
        finally:   # the instances' state as it was before tuning, whatever happened
            self._cache = None
            segs, nseg, _, _ = self._segments(self.STATE_FIELDS)
            _lib.check(self.lib.hs_segments_copy(saved.data_ptr(), segs.data_ptr(), nseg, 1, stream.cuda_stream),
                       'hs_segments_copy')
            stream.synchronize()
            for mm in self.magnets:
                mm._ctl = None
        return cs, k, t

    def resync(self):
        """Recompute every instance's incrementally updated energies from its spins
        (Magnets.resync_energies), enqueued on the current stream."""
        for mm in self.magnets:
            mm.resync_energies()

    def _chunks(self, steps, resync_every):
        """Per-instance step budgets of consecutive launches separated by resyncs."""
        left = list(steps)
        out = []
        while any(left):
            c = [min(r, resync_every) for r in left]
            out.append(c)
            left = [r - k for r, k in zip(left, c)]
        return out

    def run(self, steps, sizes=None, resync_every: int = 0, costs=None, one_cta=None, **kwargs):
        """Enqueue ``steps`` (an int or one int per instance) update steps of every instance
        without the stop rule; asynchronous. ``sizes``: optional cluster size per instance;
        ``costs``: optional expected device time per instance, which orders the work counter
        (longest first; default: the step-time model); ``one_cta``: optional flag per instance,
        run on one CTA of its group's clusters (HS_INST_ONE_CTA; the flagged instances of a
        group are claimed after the others). Each returned group's ``ns`` holds the
        device time of each of its instances (launch slot ``order[i]``) once the launch ends.
        ``resync_every``: recompute the energies from the spins after every that many steps
        (one engine launch per stretch; the FP64 resync that bounds the drift of the FP32
        increments)."""
        steps = [int(steps)] * len(self.magnets) if np.isscalar(steps) else [int(s) for s in steps]
        if resync_every and resync_every > 0:
            prepared = None
            for c in self._chunks(steps, int(resync_every)):
                prepared = self.run(c, sizes=sizes, costs=costs, one_cta=one_cta, **kwargs)
                for mm, k, total in zip(self.magnets, c, steps):
                    if k == int(resync_every):
                        mm.resync_energies()
            return prepared
        kws = [dict(kwargs) for _ in self.magnets]
        for mm, kw in zip(self.magnets, kws):
            mm._set_control(progress=0, done=0, t_max=float(kw.pop('t_max', math.inf)))
        key = (tuple(steps), tuple(sorted((k, float(v)) for k, v in kwargs.items() if k != 't_max')),
               tuple(mm._version for mm in self.magnets), tuple(id(mm) for mm in self.magnets),
               tuple(sizes) if sizes else None, tuple(one_cta) if one_cta else None, self.cluster_size,
               self.throughput)
        if self._cache is None or self._cache[0] != key:
            self._cache = (key, self._prepare(steps, kws, sizes, costs, one_cta))
        prepared = self._cache[1]
        self.launch(prepared)
        return prepared

    def capture(self, steps, sizes=None, resync_every: int = 0, **kwargs):
        """Record the launch of ``run(steps, ...)`` in a CUDA graph and return a
        :class:`CapturedRun`; each ``replay()`` advances every instance by ``steps`` again
        with no host work (the work counters are reset inside the graph). The instances'
        step controls are set before the capture; set them again (``run`` or ``capture``)
        after changing them on the host."""
        steps_l = [int(steps)] * len(self.magnets) if np.isscalar(steps) else [int(x) for x in steps]
        kws = [dict(kwargs) for _ in self.magnets]
        for mm, kw in zip(self.magnets, kws):
            mm._set_control(progress=0, done=0, t_max=float(kw.pop('t_max', math.inf)))
        chunks = self._chunks(steps_l, int(resync_every)) if resync_every and resync_every > 0 else [steps_l]
        preps = [self._prepare(c, kws, sizes) for c in chunks]
        for prepared in preps:      # occupancy queries happen outside the capture
            for p in prepared:
                self._max(p.cs)
        n_groups = max(len(p) for p in preps)
        if n_groups > 1 and len(self._streams) < n_groups:
            self._streams += [torch.cuda.Stream(self.device) for _ in range(n_groups - len(self._streams))]
        if len(chunks) > 1:
            self.resync()           # scratch buffers of the recomputes exist before the capture
            for mm in self.magnets:
                mm.check_resync()
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=side):
            for c, prepared in zip(chunks, preps):
                self.launch(prepared, stream=side)
                if len(chunks) > 1:
                    for mm, k in zip(self.magnets, c):
                        if k == int(resync_every):
                            mm.resync_energies()
        torch.cuda.current_stream(self.device).wait_stream(side)
        return CapturedRun(g, [p for prepared in preps for p in prepared], self)

    # ---------------------------------------------------------------- packed state transfer
    STATE_FIELDS = ('m', 'mm', 'C', 'E', 'Ep')

    @staticmethod
    def _field_tensor(mm: Magnets, f: str):
        if f == 'm':
            return mm._m_dev
        if f == 'mm':
            return mm._mm_dev
        if f == 'C':
            return mm._counters
        d = mm._dipolar()
        if d is None:
            return None
        return d._E if f == 'E' else d._Ep

    def state_layout(self, fields=STATE_FIELDS):
        """Layout of the packed state of ``fields`` ('m' int8 spins, 'mm' FP32 m * moment, 'C'
        HsCounters, 'E' / 'Ep' FP64 dipolar energies): [(instance, field, offset, bytes)] with
        every array at a 256-byte aligned offset, and the total size in bytes."""
        out, off = [], 0
        for i, mm in enumerate(self.magnets):
            for f in fields:
                t = self._field_tensor(mm, f)
                if t is None:
                    continue
                nb = t.numel() * t.element_size()
                out.append((i, f, off, nb))
                off += -(-nb // 256) * 256
        return out, off

    def _segments(self, fields):
        """Device table of HsSegment entries (at most HS_SEGMENT_MAX bytes each) for ``fields``,
        cached on the arrays' addresses."""
        lay, total = self.state_layout(fields)
        ptrs = tuple(self._field_tensor(self.magnets[i], f).data_ptr() for i, f, _, _ in lay)
        key = (tuple(fields), ptrs)
        c = getattr(self, '_seg_cache', {}).get(key)
        if c is None:
            rows = segment_table(lay, ptrs)
            t = torch.from_numpy(rows.view(np.uint8).copy()).pin_memory().to(self.device, non_blocking=True)
            c = (t, len(rows), total, lay)
            if not hasattr(self, '_seg_cache') or len(self._seg_cache) >= 8:
                self._seg_cache = {}          # instance sets changed: drop the old tables
            self._seg_cache[key] = c
        return c

    def _staging(self, which, nbytes):
        buf = getattr(self, '_stage_' + which, None)
        if buf is None or buf.numel() < nbytes:
            buf = torch.empty(max(nbytes, 256), dtype=torch.uint8, device=self.device)
            setattr(self, '_stage_' + which, buf)
        return buf

    def _gather(self, fields, stream):
        segs, n, total, _ = self._segments(fields)
        stage = self._staging('out', total)
        _lib.check(self.lib.hs_segments_copy(stage.data_ptr(), segs.data_ptr(), n, 0, stream), 'hs_segments_copy')
        return stage, total

    def pack_host(self, fields=STATE_FIELDS) -> torch.Tensor:
        """The instances' current device state of ``fields`` packed (layout :meth:`state_layout`)
        into a new pinned host buffer; synchronises."""
        st = torch.cuda.current_stream(self.device)
        stage, total = self._gather(fields, st.cuda_stream)
        host = torch.empty(total, dtype=torch.uint8).pin_memory()
        host.copy_(stage[:total], non_blocking=True)
        st.synchronize()
        return host

    def upload(self, host_in: torch.Tensor, in_fields=STATE_FIELDS, slot: int = 0):
        """Start the host to device copy of a packed state (pinned ``host_in``) into staging slot
        ``slot`` on the engine's copy stream, so that it overlaps the launches running on the
        compute stream; :meth:`run_from_host` with ``slot=`` then consumes it. A slot is reused
        only after the scatter that read it has run."""
        segs, n, total, lay = self._segments(in_fields)
        if host_in.numel() < total:
            raise ValueError(f'host_in holds {host_in.numel()} bytes, the layout needs {total}')
        if not hasattr(self, '_copy_stream'):
            self._copy_stream = torch.cuda.Stream(self.device)
            self._slot_free, self._slot_ready, self._slot_host = {}, {}, {}
        stage = self._staging(f'in{slot}', total)
        cs = self._copy_stream
        if slot in self._slot_free:
            cs.wait_event(self._slot_free[slot])
        with torch.cuda.stream(cs):
            stage[:total].copy_(host_in[:total], non_blocking=True)
        # the buffer belongs to the compute stream's pool but is written on the copy stream: if a
        # larger layout replaces it, its memory must not be reused before this copy has run
        stage.record_stream(cs)
        ev = torch.cuda.Event()
        ev.record(cs)
        self._slot_ready[slot], self._slot_host[slot] = ev, host_in
        return slot

    def run_from_host(self, steps, host_in: torch.Tensor | None = None, in_fields=STATE_FIELDS,
                      host_out: torch.Tensor | None = None, out_fields=('m', 'C'), sizes=None, slot: int | None = None,
                      **kwargs):
        """Load every instance's state from the packed pinned host buffer ``host_in`` (ONE host to
        device copy and one scatter kernel, hs_segments_copy), run ``steps`` like :meth:`run`,
        and gather ``out_fields`` into the pinned host buffer ``host_out`` (one gather kernel and
        ONE device to host copy). Asynchronous: synchronise the stream before reading host_out.
        With ``slot=`` the state was already sent by :meth:`upload` (the copy overlapped earlier
        work) and ``host_in`` may be omitted.
        The run controls (progress, done, t_max) come from the loaded counters; :meth:`run` writes
        only the ones that differ from what it needs."""
        st = torch.cuda.current_stream(self.device)
        segs, n, total, lay = self._segments(in_fields)
        if slot is None:
            if host_in is None or host_in.numel() < total:
                raise ValueError(f'host_in must hold the {total} bytes of the layout')
            stage = self._staging('in', total)
            stage[:total].copy_(host_in[:total], non_blocking=True)
        else:
            if slot not in getattr(self, '_slot_ready', {}):
                raise ValueError(f'nothing was uploaded to slot {slot}')
            st.wait_event(self._slot_ready.pop(slot))
            host_in = self._slot_host.pop(slot)
            stage = self._staging(f'in{slot}', total)
        _lib.check(self.lib.hs_segments_copy(stage.data_ptr(), segs.data_ptr(), n, 1, st.cuda_stream), 'hs_segments_copy')
        if slot is not None:
            ev = torch.cuda.Event()
            ev.record(st)
            self._slot_free[slot] = ev
        if 'C' in in_fields:
            # the loaded counters' run controls, read from the packed buffer in one gather
            inst = [i for i, f, _, _ in lay if f == 'C']
            offs = np.array([off for _, f, off, _ in lay if f == 'C'], dtype=np.int64)
            recs = host_in.numpy()[offs[:, None] + np.arange(_lib.COUNTERS_DTYPE.itemsize)]
            recs = recs.view(_lib.COUNTERS_DTYPE).ravel()
            for i, p, d, t in zip(inst, recs['progress'].tolist(), recs['done'].tolist(), recs['t_max'].tolist()):
                self.magnets[i]._ctl = {'progress': p, 'done': d, 't_max': t}
        prepared = self.run(steps, sizes=sizes, **kwargs)
        if host_out is not None:
            out_stage, out_total = self._gather(out_fields, st.cuda_stream)
            if host_out.numel() < out_total:
                raise ValueError(f'host_out holds {host_out.numel()} bytes, the layout needs {out_total}')
            host_out[:out_total].copy_(out_stage[:out_total], non_blocking=True)
        return prepared

    #: steps an instance makes per engine launch of progress(); an unfinished run is continued
    #: by the next launch, so no launch runs unboundedly long
    progress_launch_steps = 1 << 16

    def progress(self, t_max=1.0, MCsteps_max=4.0, **kwargs):
        """The reference's progress() for every instance at once; returns [(dt, dMCsteps)].
        Runs engine launches of at most ``progress_launch_steps`` steps per instance until every
        instance's stop rule holds."""
        from .core import check_progress_limits
        check_progress_limits(t_max, MCsteps_max)
        starts = []
        for mm in self.magnets:
            c = mm._read_counters()
            t0, mc0 = float(c['t']), float(c['attempted']) / mm.n
            mm._write_counters(t0=t0, mc0=mc0, t_max=float(t_max), mc_max=float(MCsteps_max), progress=1, done=0)
            starts.append((t0, mc0))
        budget = max(1, int(self.progress_launch_steps))
        prepared = self._prepare([budget] * len(self.magnets), [dict(kwargs) for _ in self.magnets])
        self.launches = 0
        while True:
            self.launch(prepared)
            self.launches += 1
            counters = [mm._read_counters() for mm in self.magnets]
            for c in counters:
                st = int(c['status'])
                if st:
                    for mm in self.magnets:
                        mm._write_counters(progress=0, done=0)
                    raise RuntimeError(f'device step reported status {st} (HS_ST_* bits)')
            if all(int(c['done']) for c in counters):
                break
        out = []
        for mm, c, (t0, mc0) in zip(self.magnets, counters, starts):
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

    def tune(self, mm: Magnets, steps=200, candidates=CLUSTER_SIZES, include_step_kernels=False, **kw) -> int:
        """Returns the chosen cluster size, or 0 for the per-step kernels (CUDA-graph replays),
        and configures ``mm.engine`` accordingly."""
        k = self.key(mm)
        if k not in self.cache:
            snap = mm._snapshot()
            persistent, cs0 = mm.engine.persistent, mm.engine.cluster_size
            best, best_t = None, math.inf
            cands = ([0] if include_step_kernels else []) + list(candidates)
            for cs in cands:
                mm.engine.persistent = cs != 0
                mm.engine.cluster_size = cs
                mm._engine_cache = None
                mm.run(max(steps // 10, 5), **kw)  # warm-up (captures graphs / prepares descriptors)
                torch.cuda.synchronize(mm.device)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                mm.run(steps, **kw)
                e1.record()
                torch.cuda.synchronize(mm.device)
                t = e0.elapsed_time(e1)
                mm._restore(snap)
                if t < best_t:
                    best, best_t = cs, t
            mm.engine.persistent, mm.engine.cluster_size = persistent, cs0
            self.cache[k] = best
        best = self.cache[k]
        mm.engine.persistent = best != 0
        mm.engine.cluster_size = best
        mm._cluster_size = best or None
        mm._engine_cache = None
        return best
