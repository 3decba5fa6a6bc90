"""Serving: a request loop for parameter-sweep simulations with continuous batching.

Requests (one lattice, its parameters and a step budget each) arrive over time. The
:class:`Server` admits them while device memory (an HBM budget, from each request's footprint
estimate) and instance slots allow, keeps every admitted Magnets state resident on the GPU,
and advances all admitted instances together in *rounds*: one persistent engine launch
(``hs_engine_run``, hotspice_b200/csrc/hs_engine.cu) per round, in which every instance runs a
quantum of steps sized so that each gets about the same device time (processor sharing
between the requests on the GPU), with cluster sizes planned from each request's remaining
work. Requests that arrive while a round runs are built on the
host and admitted into the next round, which is queued on the device behind the running one,
so their work overlaps with the requests already there. A request retires when its step
budget is done; its result and completion latency are recorded at that round's end.

Results do not depend on the mix: each instance draws its variates from its own Philox stream
(keyed by its seed and its own step counters on the device), and the engine runs the same
per-instance step sequence however the steps are cut into rounds and whichever cluster size
runs them, so a request gives the same final state alone and in any mix.

The scheduling policy (:class:`AdmissionQueue`, :func:`plan_quanta`, :func:`shard_requests` and
its run-time counterpart :class:`RequestDealer`,
and the engine's :func:`~hotspice_b200.engine.plan_sizes`)
is plain host code; the reference has no serving layer (its experiments call
``Magnets.progress`` in a loop, hotspice/core.py:736-760, one simulation at a time).
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from .engine import model_time, plan_sizes, step_model, step_time

LATTICE_GEOMETRY = {
    # lattice: (a, moment) of the sweep's instances
    'OOP_Square': (200e-9, 1.1e-15),
    'IP_Pinwheel': (300e-9, 1e-15),
    'IP_Kagome': (500e-9, 1e-15),
    'Ising_Square': (200e-9, 1.1e-15),   # exchange-only OOP square lattice, Wolff updates
}


@dataclass
class SimRequest:
    """One simulation: ``spec`` describes the lattice and its parameters (see
    :func:`build_magnets`), ``steps`` the update steps to run, ``arrival`` the time (s) after
    the start of the stream at which it arrives."""
    rid: int
    spec: dict
    steps: int
    arrival: float = 0.0


@dataclass
class SimResult:
    rid: int
    steps: int
    arrival: float
    admitted: float
    finished: float
    switches: int
    attempts: int
    t: float
    E_tot: float
    m_avg: float
    state: np.ndarray | None = None    # final spins (int8), when the server keeps them

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def geometry_shape(spec) -> tuple[int, int]:
    """(ny, nx) of the lattice a spec builds (IP_Kagome derives ny from nx, hotspice/ASI.py)."""
    n = int(spec['n'])
    if spec['lattice'] == 'IP_Kagome':
        return int(n / math.sqrt(3)) // 4 * 4 - 1, n
    return n, n


def footprint_bytes(spec) -> int:
    """Device bytes a request holds while resident (estimate made before it is built): per
    cell the spins, moments, FP64 energies (and perpendicular energies), E_B, temperature and
    Zeeman factors, scratch; plus the kernel windows of the dipolar cutoff."""
    ny, nx = geometry_shape(spec)
    cells = nx * ny
    per_cell = 96 if spec['lattice'] in ('IP_Pinwheel', 'IP_Kagome') else 64
    kern = 0
    if spec['lattice'] != 'Ising_Square':
        w = int(spec.get('cutoff_cells', 16)) * 4 + 1
        kern = 6 * 3 * w * w * 4
    return cells * per_cell + kern + (1 << 20)


def instance_inputs(spec):
    """Seeded start state (iid +-1) and lognormal E_B field of a spec."""
    ny, nx = geometry_shape(spec)
    g = np.random.Generator(np.random.PCG64(int(spec['seed'])))
    m0 = g.integers(0, 2, size=(ny, nx)) * 2 - 1
    EB = float(spec.get('E_B', 5.5e-20)) * g.lognormal(-0.05 ** 2 / 2, 0.05, size=(ny, nx))
    return m0, EB


def build_magnets(spec, device=None):
    """The Magnets instance of a request spec: ``lattice`` in LATTICE_GEOMETRY, ``n`` (grid
    side), ``T``, Zeeman ``B`` (T) at ``angle``, ``scheme`` ('Neel' / 'Metropolis'; Ising
    lattices use Wolff with exchange ``J``), ``seed``; dipolar cutoff of ``cutoff_cells``
    lattice constants (default 16)."""
    import hotspice_b200 as hs
    lat = spec['lattice']
    a, moment = LATTICE_GEOMETRY[lat]
    m0, EB = instance_inputs(spec)
    if lat == 'Ising_Square':
        return hs.ASI.OOP_Square(a, int(spec['n']), T=spec['T'], E_B=0.0, moment=moment, pattern=m0, PBC=True,
                                 energies=[hs.ExchangeEnergy(J=float(spec.get('J', 1e-21)))],
                                 params=hs.SimParams(UPDATE_SCHEME='Wolff', MULTISAMPLING_SCHEME='cluster'),
                                 seed=int(spec['seed']), device=device)
    cls = getattr(hs.ASI, lat)
    cut = float(spec.get('cutoff_cells', 16)) * a
    return cls(a, int(spec['n']), T=spec['T'], E_B=EB, moment=moment, pattern=m0,
               energies=[hs.DipolarEnergy(cutoff_range=cut), hs.ZeemanEnergy(spec.get('B', 0.0), spec.get('angle', 0.0))],
               params=hs.SimParams(UPDATE_SCHEME=spec.get('scheme', 'Neel')), seed=int(spec['seed']), device=device)


def request_stream(n_requests, rate=200.0, n_range=(64, 1024), steps_range=(1000, 100000), seed=7,
                   lattices=('OOP_Square', 'IP_Pinwheel', 'IP_Kagome', 'Ising_Square')):
    """Seeded Poisson arrival stream of sweep requests: exponential inter-arrival times of
    mean 1/rate, lattice uniform over ``lattices``, n and steps log-uniform over their ranges,
    T uniform in [200, 400] K, Zeeman 0-5 mT at a random angle; dipolar lattices alternate
    Néel / Metropolis."""
    g = np.random.Generator(np.random.PCG64(seed))
    t = 0.0
    out = []
    for i in range(n_requests):
        t += float(g.exponential(1.0 / rate))
        lat = lattices[int(g.integers(0, len(lattices)))]
        n = int(round(math.exp(g.uniform(math.log(n_range[0]), math.log(n_range[1])))))
        steps = int(round(math.exp(g.uniform(math.log(steps_range[0]), math.log(steps_range[1])))))
        spec = dict(lattice=lat, n=n, T=float(g.uniform(200, 400)), B=float(g.uniform(0, 5e-3)),
                    angle=float(g.uniform(0, 2 * math.pi)), scheme='Neel' if i % 2 == 0 else 'Metropolis',
                    seed=seed * 1_000_003 + i)
        out.append(SimRequest(i, spec, steps, t))
    return out


class AdmissionQueue:
    """Arrived requests wait here in arrival order; :meth:`admit` hands out those that fit
    the free device bytes and slots, first come first admitted. A request that does not fit
    yet lets later ones that do fit pass it, until it has been passed over ``max_skip`` times;
    from then on nothing behind it is admitted before it (so a large request cannot starve)."""

    def __init__(self, footprint=footprint_bytes, max_skip=64):
        self.waiting: deque[SimRequest] = deque()
        self.footprint = footprint
        self.max_skip = max_skip
        self._skipped = {}

    def push(self, req: SimRequest):
        self.waiting.append(req)

    def __len__(self):
        return len(self.waiting)

    def admit(self, free_bytes: int, free_slots: int) -> list[SimRequest]:
        out, keep = [], deque()
        blocked = False
        while self.waiting:
            r = self.waiting.popleft()
            need = self.footprint(r.spec)
            if not blocked and free_slots > 0 and need <= free_bytes:
                out.append(r)
                free_bytes -= need
                free_slots -= 1
                self._skipped.pop(r.rid, None)
                continue
            keep.append(r)
            if not blocked:
                s = self._skipped.get(r.rid, 0) + 1
                self._skipped[r.rid] = s
                if s > self.max_skip:
                    blocked = True   # the head has been bypassed long enough: admit nothing behind it
        self.waiting = keep
        return out


def plan_quanta(times, remaining, round_us, sizes=None, n_sm=None):
    """Steps each active instance runs in the next round: about ``round_us`` of device time
    (``times``: time of one step of each instance on its cluster), at least one step, at most
    what remains of its budget. With the cluster ``sizes`` and the SM count, an instance whose
    remaining run is longer than the time the resident work needs to drain (its total
    remaining SM time / SMs) gets a quantum longer in proportion, up to the length of the
    round, so that the longest requests do not end alone on an otherwise idle GPU."""
    targets = [round_us] * len(times)
    if sizes is not None and n_sm:
        rem_us = [r * t for r, t in zip(remaining, times)]
        drain = sum(x * c for x, c in zip(rem_us, sizes)) / n_sm
        W = max(round_us, sum(min(round_us, x) * c for x, c in zip(rem_us, sizes)) / n_sm)
        if drain > 0:
            targets = [min(W, max(round_us, W * x / drain)) for x in rem_us]
    out = []
    for t, r, u in zip(times, remaining, targets):
        q = max(1, int(u // max(t, 1e-9)))
        out.append(int(min(q, r)))
    return out


def shard_requests(requests, world_size, rank):
    """The requests one rank serves: greedy least-loaded assignment of the stream (in arrival
    order) by estimated work (steps x per-step cost), the same on every rank, so no
    collective is needed to agree on it."""
    load = [0.0] * world_size
    mine = []
    for r in requests:
        w = request_work(r)
        k = min(range(world_size), key=lambda j: (load[j], j))
        load[k] += w
        if k == rank:
            mine.append(r)
    return mine


def request_work(r) -> float:
    """Estimated device work of a request (the unit :func:`shard_requests` balances)."""
    ny, nx = geometry_shape(r.spec)
    return r.steps * float(nx * ny + 1089)


class RequestDealer:
    """Placement of a shared arrival stream at run time (one dealer per rank, over a
    ``torch.distributed`` key-value store that all ranks share). Requests are dealt in arrival
    order: when the next undealt request has arrived, the rank whose published load (the
    estimated work it still holds, :func:`request_work` units) is the smallest claims it, by a
    compare-and-set on the shared index; a request that has waited ``grace_s`` is claimed by
    whichever rank polls first, so a rank busy in a long round delays nobody. A rank that falls
    behind its estimate (a long request, a slow lattice) keeps a high load and receives nothing
    until it has worked it off. Store round trips are limited to one poll per ``poll_s``. The
    shared index is stored as "index:claimer", so a compare-and-set that another rank won can
    never look like this rank's own. Use a fresh ``prefix`` for every stream on a store."""

    def __init__(self, requests, store, rank, world_size, prefix='hs_dealer', grace_s=0.02, poll_s=1e-3):
        self.reqs = sorted(requests, key=lambda r: (r.arrival, r.rid))
        self.store, self.rank, self.world = store, int(rank), int(world_size)
        self.prefix, self.grace_s, self.poll_s = prefix, float(grace_s), float(poll_s)
        self.next = 0            # the shared index, as last read
        self._last_poll = -math.inf
        if self.rank == 0:
            store.set(f'{prefix}/next', '0:-1')
        store.set(f'{prefix}/load{self.rank}', '0')
        for q in range(self.world):   # every rank's load key exists before anyone reads it
            store.wait([f'{prefix}/load{q}'])
        store.wait([f'{prefix}/next'])

    def _get(self, key) -> str:
        return self.store.get(f'{self.prefix}/{key}').decode()

    def exhausted(self) -> bool:
        """Every request has been dealt (as last read from the store)."""
        return self.next >= len(self.reqs)

    def claim(self, now: float, load: float, force: bool = False) -> list:
        """The requests this rank takes at time ``now`` (s after the start of the stream;
        ``math.inf`` when every request is present from the start), given its current ``load``;
        publishes the load. Reads the store at most once per ``poll_s`` unless ``force``."""
        t = time.perf_counter()
        if self.exhausted() or (not force and t - self._last_poll < self.poll_s):
            return []
        self._last_poll = t
        self.store.set(f'{self.prefix}/load{self.rank}', repr(float(load)))
        out = []
        while True:
            val = self._get('next')
            self.next = int(val.split(':')[0])
            if self.next >= len(self.reqs) or self.reqs[self.next].arrival > now:
                break
            r = self.reqs[self.next]
            # the least-loaded rule (no grace without a clock: all requests present at once)
            if self.world > 1 and (math.isinf(now) or now - r.arrival < self.grace_s):
                loads = [float(self._get(f'load{q}')) for q in range(self.world)]
                if min(range(self.world), key=lambda q: (loads[q], q)) != self.rank:
                    break
            mine = f'{self.next + 1}:{self.rank}'
            if self.store.compare_set(f'{self.prefix}/next', val, mine).decode() == mine:
                out.append(r)
                self.next += 1
                load += request_work(r)
                self.store.set(f'{self.prefix}/load{self.rank}', repr(float(load)))
        return out


@dataclass(eq=False)
class _Active:
    req: SimRequest
    mm: object
    remaining: int
    model: tuple
    admitted: float
    bytes: int
    event: object = None         # build finished (stream event)
    since_resync: int = 0        # steps run since the energies were last recomputed
    ratio: float = 1.0           # measured / modelled device time of its quanta (running average)
    measured: bool = False

    def calibrated(self):
        """The step-time model scaled by what the request's quanta measured."""
        s0, p, alpha = self.model
        return (s0 * self.ratio, p * self.ratio, alpha)


@dataclass
class ServeStats:
    makespan: float = 0.0
    rounds: int = 0
    max_active: int = 0
    attempts: int = 0
    admitted_bytes_peak: int = 0
    # per round: (host clock s, resident, round device ms, measured SM-us of its quanta,
    # longest quantum us, device idle ms before it, host ms to plan and launch it)
    history: list = field(default_factory=list)
    build_s: float = 0.0          # host time spent building admitted requests (summed over builders)
    last_active_s: float = 0.0    # when the last request became resident (s after the start)
    round_ms_sum: float = 0.0     # device time of the rounds (two may overlap)
    sm_us_sum: float = 0.0        # modelled SM time of the rounds' quanta at their cluster sizes
    sm_us_one_cta: float = 0.0    # the same quanta modelled on one CTA each
    measured_sm_us: float = 0.0   # device time the engine measured per quantum x its CTAs


class Server:
    """Continuous-batching request loop on one GPU.

    ``hbm_budget``: device bytes the resident instances may hold (default: half of the free
    memory when the server starts); ``max_slots``: resident instances at most; ``round_ms``:
    device time one instance's quantum aims at (the engine's step-time model, scaled per request
    by the device time its past quanta measured; longer when the host's planning of a round
    would outlast the round) while requests arrive, ``tail_round_ms`` once they have all
    arrived; ``keep_state``: return the final spins; ``builders``: threads that build
    admitted requests (host set-up overlaps the device rounds; default half the host cores,
    2 to 8); ``resync_every``: recompute a request's energies from its spins
    (Magnets.resync_energies) after every that many of its steps (0: never), which bounds the
    drift of the FP32 increments; quanta are cut at those points, so they fall on the same
    steps of a request whatever the mix."""

    def __init__(self, device=None, hbm_budget=None, max_slots=4096, round_ms=5.0, keep_state=False,
                 max_inflight=2, tail_round_ms=20.0, builders=None, resync_every=0):
        import torch
        from .engine import BatchEngine  # noqa: F401  (binds the engine symbols early)
        self.torch = torch
        self.device = torch.device(device) if device is not None else torch.device('cuda', torch.cuda.current_device())
        if self.device.index is None:
            self.device = torch.device(self.device.type, torch.cuda.current_device())
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            hbm_budget = free // 2
        self.hbm_budget = int(hbm_budget)
        self.max_slots = int(max_slots)
        self.round_ms = float(round_ms)
        self.keep_state = keep_state
        self.max_inflight = max(1, int(max_inflight))
        self.n_sm = torch.cuda.get_device_properties(self.device).multi_processor_count
        self.host_us = 0.0            # host time to plan and launch a round (running average)
        self.stream = torch.cuda.Stream(self.device)
        self.retire_stream = torch.cuda.Stream(self.device)
        self.build_stream = torch.cuda.Stream(self.device)
        self.stats = ServeStats()
        self._engine = None
        self.tail_round_ms = float(tail_round_ms)
        self.resync_every = int(resync_every)
        import concurrent.futures
        import os
        if builders is None:   # building is host array work that mostly releases the GIL
            builders = max(2, min(8, (os.cpu_count() or 4) // 2))
        self.builders = int(builders)
        self._builder = concurrent.futures.ThreadPoolExecutor(max_workers=max(1, self.builders))

    # -- one round ---------------------------------------------------------------------
    def _launch_round(self, active: list[_Active], round_ms: float):
        torch = self.torch
        th = time.perf_counter()
        # per-request step times: the engine's model, scaled by the request's measured quanta
        models = [a.calibrated() for a in active]
        sizes = plan_sizes(models, [a.remaining for a in active], self.n_sm)
        times = [model_time(m, c) for m, c in zip(models, sizes)]
        rem = [a.remaining for a in active]
        steps = plan_quanta(times, rem, round_ms * 1e3, sizes, self.n_sm)
        # two rounds stay in flight, so a round's device time should cover the host's planning
        # of the next one: lengthen the quanta (up to 8x) when the resident set is too small
        dev_us = sum(s * t * c for s, t, c in zip(steps, times, sizes)) / self.n_sm
        if dev_us < 2.0 * self.host_us:
            steps = plan_quanta(times, rem, round_ms * 1e3 * min(8.0, 2.0 * self.host_us / max(dev_us, 1.0)),
                                sizes, self.n_sm)
        if self.resync_every > 0:   # a quantum ends at the request's next resync point
            steps = [min(s, self.resync_every - a.since_resync) for s, a in zip(steps, active)]
        if self._engine is None:
            from .engine import BatchEngine
            self._engine = BatchEngine([a.mm for a in active], device=self.device, throughput=True)
        else:
            self._engine.set_magnets([a.mm for a in active])
        eng = self._engine
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(self.stream):
            for a in active:
                if a.event is not None:
                    self.stream.wait_event(a.event)
                    a.event = None
            e0.record(self.stream)
            prepared = eng.run(steps, sizes=sizes, costs=[s * t for s, t in zip(steps, times)])
            # each quantum's device time, copied out behind the launch (read when the round ends)
            elapsed = []
            for p in prepared:
                h = torch.empty(p.n, dtype=torch.int64, pin_memory=True)
                h.copy_(p.ns, non_blocking=True)
                elapsed.append((p.order, p.cs, h))
            for a, s in zip(active, steps):
                a.since_resync += s
                if self.resync_every > 0 and a.since_resync == self.resync_every:
                    a.mm.resync_energies()
                    a.since_resync = 0
            e1.record(self.stream)
        for a, s in zip(active, steps):
            a.remaining -= s
        sm_us = sum(s * t * c for s, t, c in zip(steps, times, sizes))
        self.stats.sm_us_sum += sm_us
        self.stats.sm_us_one_cta += sum(s * step_time(a.mm, 1) for s, a in zip(steps, active))
        return dict(prepared=prepared, e0=e0, e1=e1, members=list(active), steps=steps, sm_us=sm_us,
                    ctas=sum(sizes), sizes=sizes, elapsed=elapsed, host_ms=self._host_time(th))

    def _host_time(self, th):
        ms = (time.perf_counter() - th) * 1e3
        self.host_us = ms * 1e3 if self.host_us == 0.0 else 0.7 * self.host_us + 0.3 * ms * 1e3
        return ms

    def _calibrate(self, rd):
        """Update each member's measured/modelled ratio from the finished round's quantum
        times (running average; the first measurement replaces the prior); returns the round's
        measured SM-us and its longest quantum (us)."""
        sm, longest = 0.0, 0.0
        for order, cs, h in rd['elapsed']:
            ns = h.numpy()
            for slot, j in enumerate(order):
                a, q = rd['members'][j], rd['steps'][j]
                if q <= 0 or ns[slot] <= 0:
                    continue
                us = float(ns[slot]) * 1e-3
                sm += us * cs
                longest = max(longest, us)
                r = min(10.0, max(0.1, us / (q * model_time(a.model, cs))))
                a.ratio = r if not a.measured else 0.5 * a.ratio + 0.5 * r
                a.measured = True
        self.stats.measured_sm_us += sm
        return sm, longest

    def _retire_begin(self, a: _Active, end_event):
        """Enqueue the summary of a finished request on the retire stream, behind the round
        that finished it: its copies and small reductions run while the next round does (the
        host does not wait on the round stream, which already holds the next round)."""
        self.retire_stream.wait_event(end_event)
        with self.torch.cuda.stream(self.retire_stream):
            return a, a.mm.summary_async(keep_state=self.keep_state)

    def _retire_end(self, a: _Active, summary, now: float, t0: float) -> SimResult:
        r = summary.result()
        c = r['counters']
        st = int(c['status'])
        if st:
            raise RuntimeError(f'request {a.req.rid}: device step reported status {st} (HS_ST_* bits)')
        return SimResult(rid=a.req.rid, steps=a.req.steps, arrival=a.req.arrival, admitted=a.admitted - t0,
                         finished=now - t0, switches=int(c['switches']), attempts=int(c['attempted']),
                         t=float(c['t']), E_tot=r['E_tot'], m_avg=r['m_avg'], state=r['state'])

    # -- the loop ----------------------------------------------------------------------
    def serve(self, requests, realtime=True, dealer: RequestDealer | None = None) -> list[SimResult]:
        """Serve ``requests`` (arrival times relative to now when ``realtime``; otherwise all
        are present at the start). With a ``dealer`` (several ranks serving one stream), the
        requests come from it instead: this rank claims arrived requests while its held work is
        the smallest (``requests`` is then ignored). Returns one SimResult per request, in
        completion order."""
        torch = self.torch
        pending = deque(sorted(requests, key=lambda r: r.arrival)) if dealer is None else deque()
        queue = AdmissionQueue()
        active: list[_Active] = []
        inflight: deque = deque()
        results: list[SimResult] = []
        used_bytes = 0
        t0 = time.perf_counter()
        st = self.stats = ServeStats()

        def clock():
            return time.perf_counter() - t0

        building: list = []      # (request, footprint, future) of admitted requests being built
        retiring: list = []      # (active record, RunSummary) of finished requests being read out
        prev_end = None          # end event of the last finished round

        def collect():
            """Turn the read-outs that have landed into results."""
            if not retiring:
                return
            now = time.perf_counter()
            still = []
            for a, sm in retiring:
                if sm.ready():
                    results.append(self._retire_end(a, sm, now, t0))
                    st.attempts += results[-1].attempts
                else:
                    still.append((a, sm))
            retiring[:] = still

        def build(r):
            # runs on the builder thread: its own stream, an event the rounds wait on
            tb = time.perf_counter()
            torch.cuda.set_device(self.device)
            with torch.cuda.stream(self.build_stream):
                mm = build_magnets(r.spec, device=self.device)
                if mm.in_plane:
                    mm._orient64()   # device orientation for the read-out of m_avg
                ev = torch.cuda.Event()
                ev.record(self.build_stream)
            st.build_s += time.perf_counter() - tb
            return mm, ev

        def admit():
            """Move arrived requests to the queue, start building those that fit (the builder
            thread works while rounds run) and activate the ones that are built."""
            nonlocal used_bytes
            now = clock()
            while pending and (not realtime or pending[0].arrival <= now):
                queue.push(pending.popleft())
            if dealer is not None and not dealer.exhausted():
                held = sum(a.remaining * request_work(a.req) / max(1, a.req.steps) for a in active) + \
                    sum(request_work(r) for r in queue.waiting) + sum(request_work(r) for r, _, _ in building)
                for r in dealer.claim(now if realtime else math.inf, held):
                    queue.push(r)
            changed = False
            if queue:
                reserved = sum(a.bytes for a in active) + sum(b for _, b, _ in building) + \
                    sum(a.bytes for a, _ in retiring)
                new = queue.admit(self.hbm_budget - reserved, self.max_slots - len(active) - len(building))
                for r in new:
                    building.append((r, footprint_bytes(r.spec), self._builder.submit(build, r)))
            still = []
            for r, b, fut in building:
                if fut.done():
                    mm, ev = fut.result()
                    active.append(_Active(r, mm, int(r.steps), step_model(mm), time.perf_counter(), b, ev))
                    st.last_active_s = clock()
                    changed = True
                else:
                    still.append((r, b, fut))
            building[:] = still
            used_bytes = sum(a.bytes for a in active) + sum(b for _, b, _ in building)
            st.admitted_bytes_peak = max(st.admitted_bytes_peak, used_bytes)
            return changed

        def dealing():
            return dealer is not None and not dealer.exhausted()

        while pending or dealing() or queue or active or inflight or building or retiring:
            admit()
            collect()
            runnable = [a for a in active if a.remaining > 0]
            if runnable and len(inflight) < self.max_inflight:
                # short rounds while requests still arrive (they join at round boundaries),
                # longer ones once the stream has ended
                rms = self.round_ms if (pending or dealing() or queue or building) else \
                    max(self.round_ms, self.tail_round_ms)
                inflight.append(self._launch_round(runnable, rms))
                st.rounds += 1
                st.max_active = max(st.max_active, len(runnable))
                continue
            if inflight:
                rd = inflight[0]
                # overlap: activate newly built requests while the oldest round runs
                while not rd['e1'].query():
                    collect()
                    if not admit():
                        time.sleep(50e-6)
                rd['e1'].synchronize()
                inflight.popleft()
                ms = rd['e0'].elapsed_time(rd['e1'])
                sm, longest = self._calibrate(rd)
                idle = prev_end.elapsed_time(rd['e0']) if prev_end is not None else 0.0
                prev_end = rd['e1']
                st.history.append((clock(), len(rd['members']), ms, sm, longest, idle, rd['host_ms']))
                st.round_ms_sum += ms
                done_ids = set()
                for a in rd['members']:
                    if a.remaining <= 0 and not any(a is m for r2 in inflight for m in r2['members']):
                        retiring.append(self._retire_begin(a, rd['e1']))
                        done_ids.add(id(a))
                if done_ids:
                    active[:] = [a for a in active if id(a) not in done_ids]
                continue
            if retiring and not building:
                retiring[0][1].event.synchronize()
                continue
            if building:
                for _, _, fut in building:
                    if fut.done():
                        break
                else:
                    time.sleep(100e-6)
                continue
            if queue and not active:
                r = queue.waiting[0]
                raise RuntimeError(f'request {r.rid} needs about {footprint_bytes(r.spec)} device bytes, more than the '
                                   f'HBM budget of {self.hbm_budget} (or max_slots={self.max_slots} is 0)')
            if pending and realtime:
                time.sleep(max(0.0, min(1e-3, pending[0].arrival - clock())))
            elif dealing():
                time.sleep(2e-4)
        st.makespan = clock()
        return results


def latency_summary(results) -> dict:
    lat = np.array([r.latency for r in results], dtype=float)
    if lat.size == 0:
        return {'p50_s': None, 'p99_s': None, 'mean_s': None}
    return {'p50_s': float(np.percentile(lat, 50)), 'p99_s': float(np.percentile(lat, 99)), 'mean_s': float(lat.mean())}


def fifo_latencies(arrivals, service_times) -> np.ndarray:
    """Completion latencies of a one-at-a-time server (first come, first served) with the
    given arrival and service times."""
    t = 0.0
    out = []
    for a, s in zip(arrivals, service_times):
        t = max(t, a) + s
        out.append(t - a)
    return np.asarray(out)
