"""Benchmark of the kinetic Monte Carlo hot path on B200.

Headline workload ("batched", the configuration the metric's batched-vs-plain comparison is
quoted on): 256 independent lattice instances, lattice drawn uniformly from {OOP square
(a = 200 nm, moment 1.1e-15), IP pinwheel (a = 300 nm, moment 1e-15), kagome (a = 500 nm,
moment 1e-15)}, grid n uniform in [32, 256], T uniform in [200, 400] K, Zeeman 0-5 mT at a
random angle, E_B lognormal (mean 5.5e-20 J, 5 % sigma), dipolar cutoff 16a, Néel-Arrhenius
for even and Metropolis (grid selection, default r = calc_r(0.05)) for odd instances, FP32
energies. Seeded synthetic inputs; no dataset is involved. One bench step advances every
instance by 200 update steps in one persistent engine launch (the full workload is 20,000
steps each, i.e. 100 bench steps).

  value : switch-attempts/s of the whole batch, state resident in HBM, L2 flushed (256 MB
          write) between bench steps.
  e2e   : the same through the public API (BatchEngine.run) with every instance's start state
          copied in from pinned host memory and the spins and counters copied out per step.
  plain : the plain single-instance GPU form (Magnets.update() once per step, one instance
          at a time) on a sample of the same instances.
  single_instance: the 512 x 512 pinwheel lattice (131,072 magnets, cutoff 20a + 1 mT Zeeman,
          Metropolis grid r = 20a, 1000 steps per bench step) with the best single-instance
          path (autotuned).

Multi-GPU: one independent batch per rank (independent instances, no data-path collective);
value = all ranks' attempts / max-over-ranks device time.

`--impl reference` times the reference algorithm's NumPy restatement (the oracle) on the host
on a bounded sample of the same instances.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "switch-attempts/sec/GPU batched-served vs plain at 1e-6 rel-E err; p50/p99 latency"
UNIT = "switch-attempts/s"
SEED = 20261203
N_INST = 256
STEPS_PER_BENCH_STEP = 200
LATTICES = (('OOP_Square', 200e-9, 1.1e-15), ('IP_Pinwheel', 300e-9, 1e-15), ('IP_Kagome', 500e-9, 1e-15))
WORKLOAD = ("batched: 256 instances, lattice uniform in {OOP_Square a=200nm, IP_Pinwheel a=300nm, IP_Kagome a=500nm}, "
            "n uniform in [32,256], T uniform in [200,400]K, Zeeman 0-5mT random angle, E_B lognormal(5.5e-20, 5%), "
            "dipolar cutoff 16a, Neel (even) / Metropolis grid (odd), 200 steps per instance per bench step, FP32")


def instance_specs(n_inst=N_INST, seed=SEED):
    g = np.random.Generator(np.random.PCG64(seed))
    specs = []
    for i in range(n_inst):
        kind = int(g.integers(0, 3))
        n = int(g.integers(32, 257))
        specs.append(dict(i=i, lattice=LATTICES[kind][0], a=LATTICES[kind][1], moment=LATTICES[kind][2], n=n,
                          T=float(g.uniform(200, 400)), B=float(g.uniform(0, 5e-3)), angle=float(g.uniform(0, 2 * math.pi)),
                          scheme='Neel' if i % 2 == 0 else 'Metropolis', seed=seed * 1000 + i))
    return specs


def _geometry_shape(spec):
    n = spec['n']
    if spec['lattice'] == 'IP_Kagome':
        return int(n / math.sqrt(3)) // 4 * 4 - 1, n
    return n, n


def instance_inputs(spec):
    ny, nx = _geometry_shape(spec)
    g = np.random.Generator(np.random.PCG64(spec['seed']))
    m0 = g.integers(0, 2, size=(ny, nx)) * 2 - 1
    EB = 5.5e-20 * g.lognormal(-0.05 ** 2 / 2, 0.05, size=(ny, nx))
    return m0, EB


def build_instance(spec, device):
    import hotspice_b200 as hs
    m0, EB = instance_inputs(spec)
    cls = getattr(hs.ASI, spec['lattice'])
    return cls(spec['a'], spec['n'], T=spec['T'], E_B=EB, moment=spec['moment'], pattern=m0,
               energies=[hs.DipolarEnergy(cutoff_range=16 * spec['a']), hs.ZeemanEnergy(spec['B'], spec['angle'])],
               params=hs.SimParams(UPDATE_SCHEME=spec['scheme']), seed=spec['seed'], device=device)


def build_oracle_instance(spec):
    from oracle import geometry as G
    from oracle.hotspice_oracle import OracleDipolar, OracleMagnets, OracleZeeman
    m0, EB = instance_inputs(spec)
    geo = {'OOP_Square': G.oop_square, 'IP_Pinwheel': G.ip_pinwheel, 'IP_Kagome': G.ip_kagome}[spec['lattice']]
    return OracleMagnets(geo(spec['a'], spec['n']), m0, T=spec['T'], E_B=EB, moment=spec['moment'],
                         energies=[OracleDipolar(cutoff_range=16 * spec['a']), OracleZeeman(spec['B'], spec['angle'])],
                         params=dict(UPDATE_SCHEME=spec['scheme']), seed=spec['seed'])


# ---------------------------------------------------------------------------- single instance
A1, N1 = 300e-9, 512
WORKLOAD1 = ("IP_Pinwheel 512x512 (131072 magnets), a=300nm, moment=1e-15, E_B lognormal(6e-20, 5%), T=300K, "
             "dipolar cutoff 20a + Zeeman 1mT@22.5deg, Metropolis grid r=20a, 1000 steps per bench step")


def build_single(device, seed=SEED):
    import hotspice_b200 as hs
    g = np.random.Generator(np.random.PCG64(seed))
    m0 = g.integers(0, 2, size=(N1, N1)) * 2 - 1
    EB = 6e-20 * g.lognormal(-0.05 ** 2 / 2, 0.05, size=(N1, N1))
    return hs.ASI.IP_Pinwheel(A1, N1, T=300.0, E_B=EB, moment=1e-15, pattern=m0,
                              energies=[hs.DipolarEnergy(cutoff_range=20 * A1), hs.ZeemanEnergy(1e-3, math.radians(22.5))],
                              params=hs.SimParams(UPDATE_SCHEME='Metropolis'), seed=seed, device=device)


# ---------------------------------------------------------------------------- plumbing
class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled during the timed region: through NVML
    every 10 ms (the timed regions here can be ~100 ms), else nvidia-smi every 200 ms."""
    Q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,'
         'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,'
         'clocks_event_reasons.sw_power_cap')
    # NVML clock-event reason bits
    BITS = (('hw_slowdown', 0x8), ('hw_thermal_slowdown', 0x40), ('sw_thermal_slowdown', 0x20), ('sw_power_cap', 0x4))

    def __init__(self, index):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None
        self._nvml = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            h = None
            try:
                pr = torch.cuda.get_device_properties(index)
                bus = f"{pr.pci_domain_id:08X}:{pr.pci_bus_id:02X}:{pr.pci_device_id:02X}.0"
                h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            except Exception:
                h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self._nvml = (pynvml, h, float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)))
        except Exception:
            self._nvml = None

    def _sample_nvml(self):
        nv, h, mx = self._nvml
        sm = float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
        try:
            bits = int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))
        except Exception:
            bits = int(nv.nvmlDeviceGetCurrentClocksThrottleReasons(h))
        flags = ['Active' if bits & b else 'Not Active' for _, b in self.BITS]
        self.rows.append([str(self.index), str(sm), str(mx), '', hex(bits)] + flags)

    def _run(self):
        while not self._stop.is_set():
            try:
                if self._nvml is not None:
                    self._sample_nvml()
                    self._stop.wait(0.01)
                    continue
                out = subprocess.run(['nvidia-smi', f'--query-gpu={self.Q}', '--format=csv,noheader,nounits',
                                      '-i', str(self.index)], capture_output=True, text=True, timeout=5).stdout
                self.rows.append([c.strip() for c in out.strip().split(',')])
            except Exception:
                self._nvml = None
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace('.', '').isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace('.', '').isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        reasons = set()
        for r in self.rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower().startswith('active'):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def dist_setup():
    ws = int(os.environ.get('WORLD_SIZE', '1'))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120))
        return dist, dist.get_rank(), ws, int(os.environ.get('LOCAL_RANK', '0'))
    return None, 0, 1, 0


def measured_peaks():
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as f:
            p = json.load(f)
        return float(p['hbm_gbs']), 'measured'
    except Exception:
        return 6650.0, 'fallback'


def profile_traffic():
    """Per-launch DRAM traffic of the engine kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, 'profiles', 'engine_kernel_batched256.txt')
    try:
        for line in open(path):
            if line.startswith('traffic_bytes_per_launch:'):
                return float(line.split(':', 1)[1])
    except OSError:
        pass
    return None


def algorithmic_bytes(mm, dattempts, dswitches, steps):
    """Bytes a step must move, from the run's own counters: a Néel step reads every occupied
    cell's FP64 energy, spin, Zeeman factor and E_B (17 B; +12 B of E_perp and its Zeeman
    factor in-plane); a Metropolis step reads those for its candidates; every switch
    read-modify-writes the FP64 energy and reads the FP32 kernel and source field over its
    window (24 B per window cell; +20 B for E_perp and its kernel in-plane)."""
    d = mm._dipolar()
    W = (2 * d.kernel_set.wx + 1) * (2 * d.kernel_set.wy + 1)
    per_cell = 17 + (12 if mm.USE_PERP_ENERGY else 0)
    upd = W * (24 + (20 if mm.USE_PERP_ENERGY else 0))
    if mm.params.UPDATE_SCHEME.name == 'NEEL':
        return steps * mm.n * per_cell + dswitches * upd
    return dattempts * per_cell + dswitches * upd


# ---------------------------------------------------------------------------- reference arm
def oracle_sample(specs, seconds_per_instance=2.5, max_steps=400):
    """Time the NumPy oracle on a few instances of the batch (two per scheme)."""
    picks = [s for s in specs if s['scheme'] == 'Neel'][:2] + [s for s in specs if s['scheme'] == 'Metropolis'][:2]
    att, secs, steps_done = 0, 0.0, 0
    for spec in picks:
        mo = build_oracle_instance(spec)
        mo.update()
        a0, t0, k = mo.attempted_switches, time.perf_counter(), 0
        while k < max_steps and time.perf_counter() - t0 < seconds_per_instance:
            mo.update()
            k += 1
        secs += time.perf_counter() - t0
        att += mo.attempted_switches - a0
        steps_done += k
    return att / secs, secs, steps_done, len(picks)


def _oracle_worker_loop(share, inq, outq):
    """One reference-arm worker process (spawned, one NumPy thread): builds the oracle
    instances of its share of the batch once, then on every ('run', k) command advances each of
    them by k steps and reports (instance, attempts, seconds, steps) per instance."""
    for var in ('OMP_NUM_THREADS', 'OPENBLAS_NUM_THREADS', 'MKL_NUM_THREADS'):
        os.environ[var] = '1'
    insts = {}
    while True:
        cmd = inq.get()
        if cmd is None:
            return
        _, k = cmd
        res = []
        for spec in share:
            mo = insts.get(spec['i'])
            if mo is None:
                mo = insts[spec['i']] = build_oracle_instance(spec)
            a0, t0 = mo.attempted_switches, time.perf_counter()
            for _ in range(k):
                mo.update()
            res.append((spec['i'], mo.attempted_switches - a0, time.perf_counter() - t0, k))
        outq.put(res)


def reference_workers():
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    return max(1, min(n, 128))


def run_reference(args):
    """The reference arm: the NumPy oracle (the reference's algorithm restated; the reference
    itself is Python that cannot travel to the machine this runs on) on all host cores, over
    the whole batch. Worker process w (one per core, one NumPy thread each, spawned) owns the
    instances i = w, w + nw, ... of the 256-instance batch; a bench step advances every instance
    of the batch by ``ref_steps`` steps. Its value is the batch's rate with the work spread over
    the workers: nw * sum_i(attempts_i / steps_i) / sum_i(seconds_i / steps_i)."""
    import multiprocessing
    rank, ws = int(os.environ.get('RANK', '0')), int(os.environ.get('WORLD_SIZE', '1'))
    if rank != 0:
        return
    specs = instance_specs()
    nw = min(reference_workers(), len(specs))
    ctx = multiprocessing.get_context('spawn')
    procs, ins, outq = [], [], ctx.Queue()
    for w in range(nw):
        q = ctx.Queue()
        p = ctx.Process(target=_oracle_worker_loop, args=(specs[w::nw], q, outq), daemon=True)
        p.start()
        procs.append(p)
        ins.append(q)

    def step(k):
        t0 = time.perf_counter()
        for q in ins:
            q.put(('run', k))
        res = [r for _ in range(nw) for r in outq.get()]
        a = sum(att / st for _, att, _, st in res)
        t = sum(sec / st for _, _, sec, st in res)
        return nw * a / t, time.perf_counter() - t0, res

    try:
        for _ in range(max(1, args.warmup)):     # builds every worker's instances
            step(1)
        vals, walls = [], []
        for _ in range(args.steps):
            v, wall, res = step(args.ref_steps)
            vals.append(v)
            walls.append(wall)
    finally:
        for q in ins:
            q.put(None)
        for p in procs:
            p.join(timeout=30)
    v = float(np.mean(vals))
    sample = (f"all {len(specs)} instances of the batch, {args.ref_steps} steps of each per bench step; "
              f"{nw} worker processes (one NumPy thread each) own 1/{nw} of the instances each; rate = "
              f"{nw} x sum(attempts per step) / sum(seconds per step) over the instances")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(walls)), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "same_config": True, "sample": sample},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": nw, "kind": "port",
                             "sample": sample + " (the NumPy oracle restating the reference)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------------------- product arm
def run_product(args):
    import torch
    from hotspice_b200.engine import BatchEngine
    dist, rank, ws, local = dist_setup()
    dev = torch.device('cuda', local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    specs = instance_specs(args.instances, seed=SEED + 7919 * rank)
    t_setup = time.perf_counter()
    mms = [build_instance(s, dev) for s in specs]
    setup_s = time.perf_counter() - t_setup
    eng = BatchEngine(mms)
    S = args.mc_steps
    # the launch plan (cluster size, which runs get whole clusters) measured on the device; the
    # instances' state is restored afterwards
    tune_cs, tune_k, tune_ms = eng.tune_split(S)

    # ---- device-resident throughput: one persistent launch per bench step, replayed from a
    # CUDA graph (BatchEngine.capture) ---------------------------------------------------------
    graph = eng.capture(S)
    for _ in range(args.warmup):
        graph.replay()
    torch.cuda.synchronize(dev)
    c0 = [mm._read_counters() for mm in mms]
    if dist:
        dist.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    sampler = ClockSampler(local)
    with sampler:
        for k in range(args.steps):
            flush.fill_(float(k))
            ev[k][0].record(stream)
            graph.replay()
            ev[k][1].record(stream)
        torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    dev_ms = sum(a.elapsed_time(b) for a, b in ev)
    c1 = [mm._read_counters() for mm in mms]
    attempts = sum(int(b['attempted'] - a['attempted']) for a, b in zip(c0, c1))
    switches = sum(int(b['switches'] - a['switches']) for a, b in zip(c0, c1))
    status = [int(b['status']) for b in c1]
    near = sum(int(b['near_threshold'] - a['near_threshold']) for a, b in zip(c0, c1))
    alg = sum(algorithmic_bytes(mm, int(b['attempted'] - a['attempted']), int(b['switches'] - a['switches']),
                                S * args.steps) for mm, a, b in zip(mms, c0, c1)) / args.steps
    launch_ms = dev_ms / args.steps
    hbm, peak_kind = measured_peaks()
    achieved = alg / (launch_ms * 1e-3) / 1e9
    cluster_sizes = sorted({p.cs for p in graph.prepared})
    one_cta = sum(p.one_cta for p in graph.prepared)

    # ---- energy error of the batch against an FP64 recompute ------------------------------
    # Only instances whose kernel is symmetric: with a pair of magnets exactly at the cutoff
    # radius the reference's kernel keeps the pair one way and drops it the other (distances
    # are cumulative sums), so its incremental energies drift from any full recompute by
    # construction (the FP64 reference algorithm drifts identically).
    errs = []
    sym = [mm for mm in mms if mm._dipolar().kernel_set.asymmetry < 1e-12]
    n_asym = len(mms) - len(sym)
    for mm in sym[:: max(1, len(sym) // 16)]:
        d = mm._dipolar()
        E32 = d._E.double().clone()
        d.update(method='direct64')
        E64 = d._E.double()
        errs.append(float((E32 - E64).abs().max() / E64.abs().max()))
        d._E.copy_(E32)

    # ---- end to end through the public API (start states in, spins + counters out) ---------
    # every bench step loads all instances' start states from one packed pinned host buffer and
    # returns their spins and counters to another (BatchEngine.run_from_host)
    IN_FIELDS, OUT_FIELDS = BatchEngine.STATE_FIELDS, ('m', 'C')
    host_in = eng.pack_host(IN_FIELDS)
    out_layout, out_total = eng.state_layout(OUT_FIELDS)
    host_out = torch.empty(out_total, dtype=torch.uint8).pin_memory()
    h2d, d2h = host_in.numel(), host_out.numel()
    cdt = _counters_dtype()
    in_layout, _ = eng.state_layout(IN_FIELDS)
    hin = host_in.numpy()
    att_in = [int(np.frombuffer(hin[o:o + nb].tobytes(), dtype=cdt)[0]['attempted']) for i, f, o, nb in in_layout if f == 'C']
    # two result buffers: step k's results are read on the host while step k + 1 runs (each
    # step still copies its own inputs in and its own results out)
    host_outs = [host_out, torch.empty(out_total, dtype=torch.uint8).pin_memory()]
    c_offs = np.array([o for i, f, o, nb in out_layout if f == 'C'], dtype=np.int64)[:, None] + np.arange(cdt.itemsize)

    def read_attempts(buf):
        return int(buf.numpy()[c_offs].view(cdt)['attempted'].sum()) - sum(att_in)

    torch.cuda.synchronize(dev)
    ee0, ee1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2e_att = 0
    ee0.record(stream)
    eng.upload(host_in, IN_FIELDS, slot=0)
    done = [None, None]
    for k in range(args.steps):
        eng.run_from_host(S, None, IN_FIELDS, host_outs[k % 2], OUT_FIELDS, slot=k % 2)
        done[k % 2] = torch.cuda.Event()
        done[k % 2].record(stream)
        if k + 1 < args.steps:      # the next step's inputs cross PCIe while this step runs
            eng.upload(host_in, IN_FIELDS, slot=(k + 1) % 2)
        if k > 0:                   # the previous step's results, read while this step runs
            done[(k - 1) % 2].synchronize()
            e2e_att += read_attempts(host_outs[(k - 1) % 2])
    done[(args.steps - 1) % 2].synchronize()
    e2e_att += read_attempts(host_outs[(args.steps - 1) % 2])
    ee1.record(stream)
    torch.cuda.synchronize(dev)
    e2e_ms = ee0.elapsed_time(ee1)

    # ---- plain single-instance GPU form on a sample of the same instances ----------------
    plain_att, plain_s, plain_n = 0, 0.0, 0
    for mm in mms[:: max(1, len(mms) // args.plain_sample)]:
        a0 = mm.attempted_switches
        t0 = time.perf_counter()
        for _ in range(args.plain_steps):
            mm.update()
        torch.cuda.synchronize(dev)
        plain_s += time.perf_counter() - t0
        plain_att += mm.attempted_switches - a0
        plain_n += 1
    plain_value = plain_att / plain_s
    plain_best = run_plain_best(mms, S, dev) if args.plain_best else None

    # ---- reductions over ranks -------------------------------------------------------------
    vals = torch.tensor([dev_ms, e2e_ms, float(attempts), float(e2e_att)], dtype=torch.float64, device=dev)
    if dist:
        mx = vals.clone(); dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        sm = vals.clone(); dist.all_reduce(sm, op=dist.ReduceOp.SUM)
        dev_ms, e2e_ms = float(mx[0]), float(mx[1])
        attempts, e2e_att = int(sm[2]), int(sm[3])
    single = None
    if rank == 0 and not args.no_single:
        single = run_single(dev, stream)
    served = None
    if args.served > 0:
        served = run_served(dev, args, dist, rank, ws)
    recompute = None
    if rank == 0 and args.recompute_n > 0:
        recompute = run_recompute(dev, n=args.recompute_n)
    incremental = None
    if rank == 0 and args.incremental_n > 0:
        incremental = run_incremental(dev, n=args.incremental_n)
    relax = None
    if rank == 0 and args.relax_n > 0:
        relax = run_relax(dev, n=args.relax_n, cpu_seconds=0.0 if args.no_cpu_baseline else 10.0)
    c3 = None
    if rank == 0 and args.c3_steps > 0:
        c3 = run_c3(dev, n=args.c3_n, steps=args.c3_steps)
    c1_run = None
    if rank == 0 and args.c1_steps > 0:
        c1_run = run_c1(dev, stream, steps=args.c1_steps, cpu_seconds=0.0 if args.no_cpu_baseline else 5.0)
    reservoir = None
    if rank == 0 and args.reservoir_n > 0:
        reservoir = run_reservoir(dev, n=args.reservoir_n, cpu_seconds=0.0 if args.no_cpu_baseline else 10.0)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    value = attempts / (dev_ms * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded lattices, random starts, lognormal E_B)",
        "config": {"workload": WORKLOAD, "instances": len(mms), "steps_per_instance_per_bench_step": S,
                   "l2": "flushed (256 MB write) between bench steps",
                   "launch": "one persistent engine launch per bench step, replayed from a CUDA graph",
                   "parallelism": f"{ws} independent batches (one per GPU)" if ws > 1 else "one batch, one GPU",
                   "cluster_sizes": cluster_sizes,
                   "instances_on_one_cta": one_cta,
                   "launch_plan": f"autotuned (BatchEngine.tune_split): the {tune_k} longest runs on clusters of "
                                  f"{tune_cs} CTAs, the rest on one CTA each ({tune_ms:.2f} ms per launch while tuning)", "switches": switches, "attempts": attempts,
                   "device_status_nonzero": sum(1 for s in status if s),
                   "near_threshold_decisions": near, "decisions": attempts,
                   "near_threshold_note": "decisions (Neel argmins, Metropolis acceptances) whose FP32 margin was "
                                          "below the effect of a 1e-6 relative energy error; counted on the device",
                   "max_rel_energy_error_vs_fp64": max(errs),
                   "energy_error_note": f"FP32 incremental vs FP64 full recompute over {len(errs)} instances with "
                                        f"symmetric kernels; {n_asym} of {len(mms)} instances have a cutoff-boundary "
                                        f"asymmetric kernel whose incremental energies drift from a full recompute in "
                                        f"the reference algorithm itself",
                   "setup_s": setup_s},
        "e2e": {"value": e2e_att / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "api": "BatchEngine.upload + run_from_host: all start states in one packed pinned buffer (one copy, "
                       "overlapping the previous step's launch, + a scatter kernel), spins + counters back the same way "
                       "into one of two pinned buffers; a step's results are read on the host while the next step runs"},
        "plain": {"value": plain_value, "unit": UNIT, "instances": plain_n, "steps_each": args.plain_steps,
                  "form": "Magnets.update() per step (host-synchronised), one instance at a time",
                  "batched_over_plain": value / plain_value},
        "gpu_launches": args.steps,
        "roofline": {"bound": "hbm", "kernel": "engine_kernel<CS> (all cluster-size groups of one bench step)",
                     "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                     "traffic": profile_traffic(), "launch_ms": launch_ms, "algorithmic_bytes_per_launch": alg},
        "clocks": sampler.summary(),
    }
    if plain_best is not None:
        plain_best["batched_over_plain_best"] = value / plain_best["value"]
        plain_best["e2e_over_plain_best"] = line["e2e"]["value"] / plain_best["value"]
        line["plain_best"] = plain_best
    if single is not None:
        line["single_instance"] = single
    if served is not None:
        line["served"] = served
    if recompute is not None:
        line["full_recompute"] = recompute
    if incremental is not None:
        line["incremental_update"] = incremental
    if relax is not None:
        line["relax"] = relax
    if reservoir is not None:
        line["reservoir"] = reservoir
    if c3 is not None:
        line["c3_poisson_resync"] = c3
    if c1_run is not None:
        line["c1_neel"] = c1_run
    if not args.no_cpu_baseline:
        v, secs, st, ni = oracle_sample(specs, seconds_per_instance=args.cpu_seconds)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
                                "sample": f"{ni} instances of the batch ({st} steps, {secs:.1f} s) with the NumPy oracle "
                                          f"restating the reference"}
    print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


def run_plain_best(mms, S, dev, tune_steps=100):
    """The best plain single-instance GPU form on the same instances: every instance alone,
    one after the other, through Magnets.run(S) on its fastest single-instance path (the
    Autotuner times the persistent engine at each cluster size and the CUDA-graph-replayed
    per-step kernels on the instance itself and keeps the fastest); the run of each is timed
    with CUDA events after a warm-up run, and the times add up (one instance at a time)."""
    import torch
    from hotspice_b200.engine import Autotuner
    tuner = Autotuner()
    att, ms, paths = 0, 0.0, {}
    for mm in mms:
        choice = tuner.tune(mm, steps=tune_steps, include_step_kernels=True)
        paths[choice] = paths.get(choice, 0) + 1
        mm.run(S)
        torch.cuda.synchronize(dev)
        a0 = mm.attempted_switches
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        mm.run(S)
        e1.record()
        torch.cuda.synchronize(dev)
        ms += e0.elapsed_time(e1)
        att += mm.attempted_switches - a0
    return {"value": att / (ms * 1e-3), "unit": UNIT, "instances": len(mms), "steps_each": S,
            "ms_total": ms, "attempts": att,
            "paths": {("per-step kernels (CUDA graphs)" if k == 0 else f"engine cluster {k}"): v
                      for k, v in sorted(paths.items())},
            "form": "Magnets.run(S) on each instance alone, one after the other, on its autotuned fastest "
                    "single-instance path (persistent engine at the best cluster size, or CUDA-graph-replayed "
                    "per-step kernels); device time summed"}


def measured_tensor_peak():
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as f:
            p = json.load(f)
        return float(p['bf16_tflops_sustained']), float(p['bf16_tflops']), 'measured'
    except Exception:
        return 1400.0, 1590.0, 'fallback'


def igemm_mma_flops(nx, ny, nsplit, BM=128, BN=256, BK=64):
    """FLOPs the implicit GEMM issues on the tensor cores for one full recompute (tiles of
    128 columns x 256 rows, every kernel row that reaches the tile, 64-column K-blocks)."""
    P = -(-nx // BM) * BM
    C = P // BK
    tot = 0
    for yt in range(-(-ny // BN)):
        y0 = yt * BN
        dlo, dhi = max(-(ny - 1), -(y0 + BN - 1)), ny - 1 - y0
        tot += (dhi - dlo + 1) * C * (P // BM)
    return tot * nsplit * 2 * BM * BN * BK


def run_recompute(dev, n=2048, n_check=512, reps=3):
    """Full dipolar recompute of an OOP square lattice with the full (uncut) kernel: the
    tensor-core implicit GEMM timed at n x n, its error against the FP64 direct sum at n_check."""
    import torch
    import hotspice_b200 as hs

    def build(k):
        g = np.random.Generator(np.random.PCG64(SEED + k))
        m0 = g.integers(0, 2, size=(k, k)) * 2 - 1
        return hs.ASI.OOP_Square(200e-9, k, T=300.0, E_B=5e-20, moment=1.1e-15, pattern=m0,
                                 energies=[hs.DipolarEnergy()], engine=hs.EngineConfig(recompute='direct64'),
                                 seed=SEED + k, device=dev)
    out = {}
    mm = build(n_check)
    d = mm._dipolar()
    d.update(method='direct64')
    E64 = d.E
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    d.update(method='direct64')
    e1.record()
    torch.cuda.synchronize(dev)
    t_direct = e0.elapsed_time(e1)
    d.update(method='igemm')
    err = float((d.E - E64).abs().max() / E64.abs().max())
    etot = abs(d.E_tot - float(E64.sum()) / 2) / abs(float(E64.sum()) / 2)
    e0.record()
    d.update(method='igemm')
    e1.record()
    torch.cuda.synchronize(dev)
    t_ig_check = e0.elapsed_time(e1)
    del mm, d, E64
    torch.cuda.empty_cache()
    mm = build(n)
    d = mm._dipolar()
    nsplit = mm.engine.igemm_splits
    d.update(method='igemm')
    torch.cuda.synchronize(dev)
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        d.update(method='igemm')
        e1.record()
        torch.cuda.synchronize(dev)
        ts.append(e0.elapsed_time(e1))
    ms = float(np.median(ts))
    fl = igemm_mma_flops(n, n, nsplit)
    sus, burst, kind = measured_tensor_peak()
    cells = n * n
    alg = 2.0 * cells * cells * (2 if mm.USE_PERP_ENERGY else 1)   # 2 N^2 per energy channel
    out.update({
        "workload": f"OOP_Square {n}x{n} ({cells} magnets), full uncut dipolar kernel ({2*n-1}x{2*n-1}), random +-1 spins; "
                    f"one full E_dipolar recompute (hs_dipolar_full_igemm, {nsplit} BF16 kernel splits, FP32 TMEM "
                    f"accumulation in chunks flushed to FP64, near field summed in FP64)",
        "ms": ms, "pairs_per_s": cells * cells / (ms * 1e-3),
        "roofline": {"bound": "tensor", "kernel": "igemm_kernel", "achieved": alg / (ms * 1e-3) / 1e12,
                     "peak": burst, "unit": "TFLOP/s", "frac": alg / (ms * 1e-3) / 1e12 / burst,
                     "peak_kind": f"{kind} bf16_tflops (burst: the recompute is timed alone; sustained {sus})",
                     "flops": "algorithmic: 2 N^2 per energy channel (N cells; every (target, source) pair one "
                              "multiply-add); the whole call is timed, its split/spin preparation and FP64 finalize "
                              "included"},
        "issued": {"tflops": fl / (ms * 1e-3) / 1e12, "flops_per_recompute": fl, "over_algorithmic": fl / alg,
                   "frac_of_burst": fl / (ms * 1e-3) / 1e12 / burst,
                   "what": f"MMA FLOPs issued on the tensor cores: {nsplit} BF16 kernel splits, padded 128 x 256 "
                           f"tiles, every kernel row that reaches a tile"},
        "check": {"n": n_check, "max_rel_err_vs_fp64_direct": err, "rel_err_E_tot": etot,
                  "igemm_ms": t_ig_check, "fp64_direct_ms": t_direct, "speedup": t_direct / t_ig_check},
    })
    del mm, d
    torch.cuda.empty_cache()
    return out


ROT_STATES = 4   # lattice states the incremental-update timing takes in turn (4 x 84 MB > L2)


def run_incremental(dev, n=2048, reps=20):
    """(a) The incremental dipolar update (hs_dipolar_update, update_multiple semantics) on an
    IP_Pinwheel n x n lattice with a 20a cutoff (81 x 81 windows, perpendicular channel on),
    timed alone through the C ABI: switches on a grid of disjoint windows (every window cell
    written once: algorithmic bytes = bytes that must move) and on the Metropolis grid spacing
    r = 20a (windows overlap; the gather still writes each cell once)."""
    import ctypes
    import torch
    import hotspice_b200 as hs
    from hotspice_b200 import _lib
    g = np.random.Generator(np.random.PCG64(SEED + 1))
    m0 = g.integers(0, 2, size=(n, n)) * 2 - 1
    mm = hs.ASI.IP_Pinwheel(A1, n, T=300.0, E_B=6e-20, moment=1e-15, pattern=m0,
                            energies=[hs.DipolarEnergy(cutoff_range=20 * A1), hs.ZeemanEnergy(1e-3, math.radians(22.5))],
                            params=hs.SimParams(UPDATE_SCHEME='Metropolis'), seed=SEED, device=dev)
    d = mm._dipolar()
    ks = d.kernel_set
    W = (2 * ks.wx + 1) * (2 * ks.wy + 1)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    lib = _lib.load()
    stream = torch.cuda.current_stream(dev).cuda_stream
    out = {"workload": f"IP_Pinwheel {n}x{n} ({n * n // 2} magnets), a=300nm, dipolar cutoff 20a "
                       f"(window {2 * ks.wx + 1}x{2 * ks.wy + 1}), perpendicular energy on, FP64 energy accumulators",
           "bytes_per_window_cell": 28}
    hbm, kind = measured_peaks()
    for label, spacing in (("disjoint windows", 2 * ks.wx + 2), ("grid spacing r=20a", 40)):
        ys, xs = np.meshgrid(np.arange(0, n - 1, spacing), np.arange(0, n - 1, spacing), indexing='ij')
        ys, xs = ys.ravel(), xs.ravel()
        xs = xs + ((ys + xs) % 2 == 0)            # pinwheel occupation: (x + y) odd
        k = len(ys)
        t, sl = mm._switch_list(k)
        t[0, :k].copy_(torch.as_tensor(ys, dtype=torch.int32))
        t[1, :k].copy_(torch.as_tensor(xs, dtype=torch.int32))
        t[2, :k].zero_()                            # exact windows
        L = mm._lattice_struct(d)
        for _ in range(3):
            _lib.check(lib.hs_dipolar_update(ctypes.byref(L), ctypes.byref(sl), None, k, _lib.HS_UPDATE_MULTIPLE, None,
                                             stream), 'hs_dipolar_update')
        torch.cuda.synchronize(dev)
        # L2 flushed (a 256 MB write) before every timed launch: the lattice's energies (84 MB)
        # would otherwise stay in the 126 MB L2 between launches
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        for e0, e1 in ev:
            flush.fill_(1.0)
            e0.record()
            lib.hs_dipolar_update(ctypes.byref(L), ctypes.byref(sl), None, k, _lib.HS_UPDATE_MULTIPLE, None, stream)
            e1.record()
        torch.cuda.synchronize(dev)
        us_flushed = sum(a.elapsed_time(b) for a, b in ev) * 1e3 / reps
        # Inputs larger than L2 instead of a flush: ROT lattice states (energies, perpendicular
        # energies, moments: 4 x 84 MB) taken in turn, so each launch reads a state last touched
        # ROT - 1 launches ago. The flush leaves the L2 full of the flush buffer's dirty lines,
        # whose write-back then shares the DRAM bus with the timed launch; with rotating states
        # the only write-back is the update's own energies, as in a run of many steps.
        states = []
        for _ in range(ROT_STATES):
            Lr = _lib.HsLattice.from_buffer_copy(L)
            keep = [d._E.clone(), mm._mm_dev.clone()]
            Lr.E_dip, Lr.mm = keep[0].data_ptr(), keep[1].data_ptr()
            if d._Ep is not None:
                keep.append(d._Ep.clone())
                Lr.E_dip_perp = keep[-1].data_ptr()
            states.append((Lr, keep))
        for j in range(2 * ROT_STATES):
            lib.hs_dipolar_update(ctypes.byref(states[j % ROT_STATES][0]), ctypes.byref(sl), None, k,
                                  _lib.HS_UPDATE_MULTIPLE, None, stream)
        torch.cuda.synchronize(dev)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
        for j, (e0, e1) in enumerate(ev):
            e0.record()
            lib.hs_dipolar_update(ctypes.byref(states[j % ROT_STATES][0]), ctypes.byref(sl), None, k,
                                  _lib.HS_UPDATE_MULTIPLE, None, stream)
            e1.record()
        torch.cuda.synchronize(dev)
        us = sum(a.elapsed_time(b) for a, b in ev) * 1e3 / reps
        del states
        alg = k * W * 28
        out[label] = {"switches": int(k), "us_per_launch": us, "window_cells_per_s": k * W / (us * 1e-6),
                      "roofline": {"bound": "hbm", "kernel": "dip_update_persist_kernel<4>" if k <= 4096 else "dip_update_kernel<4>", "achieved": alg / (us * 1e-6) / 1e9,
                                   "peak": hbm, "unit": "GB/s", "frac": alg / (us * 1e-6) / 1e9 / hbm,
                                   "peak_kind": f"{kind} hbm_gbs"},
                      "l2": f"inputs larger than L2: {ROT_STATES} lattice states ({ROT_STATES} x 84 MB) taken in turn",
                      "flushed": {"us_per_launch": us_flushed, "frac": alg / (us_flushed * 1e-6) / 1e9 / hbm,
                                  "l2": "flushed (256 MB write) before every timed launch"}}
    del mm, d, flush
    torch.cuda.empty_cache()
    return out


C3_WORKLOAD = ("OOP_Square {n}x{n} ({cells} magnets), a=200nm, moment=1.1e-15, E_B=5e-20 J, full uncut dipolar "
               "kernel, random +-1 start, Metropolis with Poisson-disc multisampling (r = calc_r(0.05), cell units), "
               "T = {temps} K, {steps} steps each, full recompute every {resync} steps as the tensor-core implicit GEMM "
               "(3 BF16 splits, FP32 accumulation, FP64 near field and finalize)")


def run_c3(dev, n=2048, steps=5000, resync=100, temps=(250.0, 300.0, 350.0)):
    """The c3 workload: per temperature, `steps` Metropolis steps with Poisson-disc selection on
    the full-kernel OOP square lattice, the energies recomputed by the tensor-core GEMM after
    every `resync` steps. Reported per temperature: step time (Poisson sampling, acceptance and
    the windowed update), recompute time, and the drift each resync removed (max |E_incremental
    - E_recomputed| / max |E|)."""
    import torch
    import hotspice_b200 as hs
    out = {"workload": C3_WORKLOAD.format(n=n, cells=n * n, temps='/'.join(f'{t:g}' for t in temps), steps=steps,
                                          resync=resync), "temperatures": {}}
    for T in temps:
        mm = hs.ASI.OOP_Square(200e-9, n, T=T, E_B=5e-20, moment=1.1e-15, pattern='random', seed=SEED + int(T),
                               energies=[hs.DipolarEnergy()], engine=hs.EngineConfig(recompute='igemm'),
                               params=hs.SimParams(UPDATE_SCHEME='Metropolis', MULTISAMPLING_SCHEME='Poisson'),
                               device=dev)
        from hotspice_b200.engine import Autotuner
        path = Autotuner().tune(mm, steps=50, include_step_kernels=True)   # fastest single-instance path
        mm.run(10)            # warm-up: graphs, scratch
        mm.resync_energies()
        mm.check_resync()
        torch.cuda.synchronize(dev)
        a0 = mm.attempted_switches
        run_ms, rec_ms, drifts = 0.0, 0.0, []
        done = 0
        while done < steps:
            k = min(resync, steps - done)
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record()
            mm.run(k)
            e1.record()
            drift = mm.resync_energies(measure=True) if k == resync else None
            e2.record()
            torch.cuda.synchronize(dev)
            run_ms += e0.elapsed_time(e1)
            if drift is not None:
                rec_ms += e1.elapsed_time(e2)
                drifts.append(drift)
            done += k
        mm.check_resync()
        att = mm.attempted_switches - a0
        out["temperatures"][f"{T:g}"] = {
            "path": "per-step kernels (CUDA graphs)" if path == 0 else f"engine cluster {path}",
            "steps": steps, "attempts": att, "switches": mm.switches, "step_us": run_ms * 1e3 / steps,
            "attempts_per_s": att / (run_ms * 1e-3), "recomputes": len(drifts),
            "recompute_ms_mean": rec_ms / max(len(drifts), 1),
            "attempts_per_s_with_recomputes": att / ((run_ms + rec_ms) * 1e-3),
            "drift_before_resync_max": max(drifts) if drifts else None,
            "drift_before_resync_median": float(np.median(drifts)) if drifts else None,
            "drift_after_resync": 0.0}
        del mm
        torch.cuda.empty_cache()
    return out


def run_relax(dev, n=1024, cpu_n=128, cpu_seconds=10.0):
    """relax() (f2): _minimize_all sweeps until the stop rule, on an IP_Pinwheel n x n from a
    random start (dipolar cutoff 8.3a, Zeeman), all on the device. CPU baseline: whole
    _minimize_all sweeps of the NumPy oracle (the reference's algorithm) on a cpu_n x cpu_n
    lattice, as magnet-sweeps per second."""
    import torch
    import hotspice_b200 as hs
    g = np.random.Generator(np.random.PCG64(SEED + 3))
    m0 = g.integers(0, 2, size=(n, n)) * 2 - 1
    mm = hs.ASI.IP_Pinwheel(A1, n, T=300.0, E_B=6e-20, moment=1e-15, pattern=m0,
                            energies=[hs.DipolarEnergy(cutoff_range=8.3 * A1), hs.ZeemanEnergy(2e-4, 0.3)],
                            seed=SEED, device=dev)
    mm.relax()                        # warm-up: builds and caches the graphs
    mm.m = m0
    mm.update_energy()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sw0 = mm.switches
    e0.record()
    mm.relax()
    e1.record()
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1)
    sweeps = mm.relax_sweeps
    out = {"workload": f"relax() of IP_Pinwheel {n}x{n} ({mm.n} magnets), a=300nm, dipolar cutoff 8.3a, Zeeman 0.2 mT, "
                       f"random start", "sweeps": sweeps, "switches": mm.switches - sw0, "ms": ms,
           "ms_per_sweep": ms / max(sweeps, 1), "magnet_sweeps_per_s": mm.n * sweeps / (ms * 1e-3)}
    del mm
    torch.cuda.empty_cache()
    # CPU: the oracle's _minimize_all on a smaller lattice (bounded sample)
    from oracle import geometry as G
    from oracle.hotspice_oracle import OracleDipolar, OracleMagnets, OracleZeeman
    geo = G.ip_pinwheel(A1, cpu_n, cpu_n)
    mc = g.integers(0, 2, size=(cpu_n, cpu_n)) * 2 - 1
    mo = OracleMagnets(geo, mc, T=300.0, E_B=6e-20, moment=1e-15, seed=SEED,
                       energies=[OracleDipolar(cutoff_range=8.3 * A1), OracleZeeman(2e-4, 0.3)])
    t0 = time.perf_counter()
    k = 0
    while time.perf_counter() - t0 < cpu_seconds and k < 50:
        mo.minimize_all()
        k += 1
    secs = time.perf_counter() - t0
    out["cpu_baseline"] = {"value": mo.n * k / secs, "unit": "magnet-sweeps/s", "cores": 1, "kind": "port",
                           "sample": f"{k} _minimize_all sweeps of IP_Pinwheel {cpu_n}x{cpu_n} with the NumPy oracle "
                                     f"({secs:.1f} s)"}
    out["gpu_over_cpu"] = out["magnet_sweeps_per_s"] / out["cpu_baseline"]["value"]
    return out


def run_reservoir(dev, n=256, inputs=20, batch=64, batch_n=128, cpu_n=64, cpu_seconds=10.0):
    """Reservoir I/O stepping (f3): OOP_Square reservoirs (dipolar cutoff 8.3a, Metropolis grid)
    driven by binary sequences through OOPSquareChessFieldInputter and read by
    OOPSquareChessOutputReader(8, 8) after every input.
    single:  one n x n reservoir, 1 MC step per input; run_sequence (field, progress() and
             readout enqueued on the device, one synchronisation) against the per-input public
             API (Inputter.input + read_state, synchronising per input);
    batched: `batch` reservoirs of batch_n x batch_n, 0.25 MC steps per input, run_batch (one
             persistent engine launch per input for all of them) against run_sequence of 4 of
             them one after the other, scaled to the batch;
    cpu:     the NumPy oracle's restatement of the reference loop on a cpu_n x cpu_n lattice."""
    import torch
    import hotspice_b200 as hs
    from hotspice_b200 import io as hio
    g = np.random.Generator(np.random.PCG64(SEED + 5))

    def make(nn, seed=SEED):
        return hs.ASI.OOP_Square(200e-9, nn, T=300, E_B=5e-20, moment=1.1e-15, pattern='random', seed=seed, device=dev,
                                 energies=[hs.DipolarEnergy(cutoff_range=8.3 * 200e-9), hs.ZeemanEnergy(0)],
                                 params=hs.SimParams(UPDATE_SCHEME='Metropolis'))

    def timed(fn):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        r = fn()
        torch.cuda.synchronize(dev)
        return r, time.perf_counter() - t0
    out = {"workload": f"OOP_Square reservoirs, dipolar cutoff 8.3a, Metropolis grid, OOPSquareChessFieldInputter 0.8 mT, "
                       f"OOPSquareChessOutputReader 8x8; single {n}x{n} x {inputs} inputs of 1 MC step; batched "
                       f"{batch} x {batch_n}x{batch_n} x {inputs} inputs of 0.25 MC step"}
    vals = (g.random(inputs) > 0.5).astype(int)
    inp = hio.OOPSquareChessFieldInputter(hio.RandomBinaryDatastream(), magnitude=8e-4, n=1, frequency=1)
    a = make(n)
    rd = hio.OOPSquareChessOutputReader(8, 8, a)
    hio.run_sequence(a, inp, vals[:2], rd)             # warm-up (descriptors)
    att0 = a.attempted_switches
    _, wall = timed(lambda: hio.run_sequence(a, inp, vals, rd))
    mc = (a.attempted_switches - att0) / a.n
    b = make(n)
    rb = hio.OOPSquareChessOutputReader(8, 8, b)
    inp.input(b, values=vals[:2])

    def api():
        for v in vals:
            inp.input(b, values=[v])
            rb.read_state(b)
    _, wall_b = timed(api)
    out["single"] = {"run_sequence_inputs_per_s": inputs / wall, "per_input_api_inputs_per_s": inputs / wall_b,
                     "magnet_mcsteps_per_s": a.n * mc / wall}
    del a, b
    # many reservoirs at once
    inq = hio.OOPSquareChessFieldInputter(hio.RandomBinaryDatastream(), magnitude=8e-4, n=0.25, frequency=1)
    bv = (g.random((batch, inputs)) > 0.5).astype(int)
    mms = [make(batch_n, SEED + 1 + i) for i in range(batch)]
    rds = [hio.OOPSquareChessOutputReader(8, 8, mm) for mm in mms]
    hio.run_batch(mms, inq, bv[:, :1], rds)           # warm-up
    att0 = sum(mm.attempted_switches for mm in mms)
    _, wall_batch = timed(lambda: hio.run_batch(mms, inq, bv, rds))
    mcs = sum(mm.attempted_switches for mm in mms) - att0
    k = 4
    seq = [make(batch_n, SEED + 1 + i) for i in range(k)]
    for mm in seq:
        hio.run_sequence(mm, inq, bv[0, :1], hio.OOPSquareChessOutputReader(8, 8, mm))
    t_seq = 0.0
    for i, mm in enumerate(seq):
        _, w = timed(lambda: hio.run_sequence(mm, inq, bv[i], hio.OOPSquareChessOutputReader(8, 8, mm)))
        t_seq += w
    out["batched"] = {"reservoirs": batch, "wall_s": wall_batch, "reservoir_inputs_per_s": batch * inputs / wall_batch,
                      "magnet_mcsteps_per_s": mcs / wall_batch,
                      "sequential_wall_s_estimate": t_seq * batch / k,
                      "batch_over_sequential": t_seq * batch / k / wall_batch}
    del mms, seq
    torch.cuda.empty_cache()
    if cpu_seconds > 0:
        from oracle import geometry as G
        from oracle.hotspice_oracle import OracleDipolar, OracleMagnets, OracleZeeman, io_input, io_read
        geo = G.oop_square(200e-9, cpu_n, cpu_n)
        mc0 = np.random.Generator(np.random.PCG64(SEED)).integers(0, 2, size=(cpu_n, cpu_n)) * 2 - 1
        mo = OracleMagnets(geo, mc0, T=300.0, E_B=5e-20, moment=1.1e-15, seed=SEED,
                           energies=[OracleDipolar(cutoff_range=8.3 * 200e-9), OracleZeeman(0.0)],
                           params=dict(UPDATE_SCHEME='Metropolis'))
        t0 = time.perf_counter()
        k = 0
        while time.perf_counter() - t0 < cpu_seconds and k < inputs:
            io_input(mo, 'chess', dict(magnitude=8e-4, n=1, frequency=1), int(vals[k]))
            io_read(mo, 'chess', dict(nx=8, ny=8))
            k += 1
        secs = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": mo.n * mo.MCsteps / secs, "unit": "magnet-MCsteps/s", "cores": 1, "kind": "port",
                               "sample": f"{k} inputs on OOP_Square {cpu_n}x{cpu_n} with the NumPy oracle ({secs:.1f} s)"}
        out["batched_over_cpu"] = out["batched"]["magnet_mcsteps_per_s"] / out["cpu_baseline"]["value"]
    return out


SERVED_WORKLOAD = ("served: the first {k} requests of a seeded Poisson arrival stream (mean 200/s); lattice uniform over "
                   "{{OOP_Square a=200nm, IP_Pinwheel a=300nm, IP_Kagome a=500nm, exchange-only square Ising J=1e-21 J "
                   "(Wolff)}}, n log-uniform in [64,1024], steps log-uniform in [1e3,1e5], T uniform in [200,400]K, Zeeman "
                   "0-5mT random angle, E_B lognormal(5.5e-20, 5%), dipolar cutoff 16a, Neel / Metropolis alternating")


OCCUPANCY = {'OOP_Square': 1.0, 'Ising_Square': 1.0, 'IP_Pinwheel': 0.5, 'IP_Kagome': 0.375}


def modelled_alone_us(spec, steps):
    """Modelled device time of a request run alone (engine step-time model at the cluster size
    the engine gives a lone instance), from its spec without building it."""
    from types import SimpleNamespace
    from hotspice_b200 import engine as E
    from hotspice_b200 import serving as SV
    from hotspice_b200.core import Scheme
    ny, nx = SV.geometry_shape(spec)
    sch = Scheme.WOLFF if spec['lattice'] == 'Ising_Square' else \
        (Scheme.NEEL if spec.get('scheme', 'Neel') == 'Neel' else Scheme.METROPOLIS)
    fake = SimpleNamespace(nx=nx, ny=ny, n=int(nx * ny * OCCUPANCY[spec['lattice']]),
                           params=SimpleNamespace(UPDATE_SCHEME=sch))
    return steps * E.step_time(fake, E.cluster_size_for(fake))


def run_served(dev, args, dist, rank, ws, sample=32):
    """Continuous batching of the c5 Poisson stream (first `args.served` requests) against
    one-request-at-a-time solves on the same arrivals. One at a time: a seeded sample of
    `sample` requests is run to completion alone through Magnets.run (the lone-instance engine
    launch), timed with CUDA events; the other requests' service times are the engine's step-time
    model for a lone instance, scaled by the sample's measured / modelled ratio."""
    import torch
    from hotspice_b200 import serving as SV
    reqs = SV.request_stream(args.served, rate=200.0, seed=SEED)
    dealer = None
    if ws > 1 and args.served_placement == 'dynamic':
        # run-time placement: each rank claims arrived requests while it holds the least work
        import datetime
        store = dist.TCPStore(os.environ.get('MASTER_ADDR', '127.0.0.1'), int(os.environ['MASTER_PORT']) + 1, ws,
                              rank == 0, timeout=datetime.timedelta(seconds=120))
        dealer = SV.RequestDealer(reqs, store, rank, ws)
        mine = []
    else:
        mine = SV.shard_requests(reqs, ws, rank) if ws > 1 else reqs
    srv = SV.Server(device=dev)
    torch.cuda.synchronize(dev)
    torch.cuda.reset_peak_memory_stats(dev)
    if dist:
        dist.barrier()
    res = srv.serve(mine, realtime=True, dealer=dealer)
    if dealer is not None:   # the requests this rank served, for its one-at-a-time baseline
        by_id = {r.rid: r for r in reqs}
        mine = sorted((by_id[x.rid] for x in res), key=lambda r: r.arrival)
    torch.cuda.synchronize(dev)
    peak_alloc = torch.cuda.max_memory_allocated(dev)
    hist = np.asarray(srv.stats.history, dtype=float).reshape(-1, 7)
    # (clock s, resident, round ms, measured SM-us, longest quantum us, idle ms before, host ms)
    rounds_diag = None
    if len(hist):
        busy = hist[:, 2] > 0
        rounds_diag = {
            "sm_use_median": float(np.median(hist[busy, 3] / (hist[busy, 2] * 1e3 * srv.n_sm))),
            "longest_quantum_over_round_median": float(np.median(hist[busy, 4] / (hist[busy, 2] * 1e3))),
            "device_idle_between_rounds_s": float(hist[:, 5].sum() * 1e-3),
            "host_ms_per_round_median": float(np.median(hist[:, 6])),
            "round_ms_median": float(np.median(hist[:, 2]))}
    mid = hist[(hist[:, 0] > 0.25 * srv.stats.makespan) & (hist[:, 0] < 0.75 * srv.stats.makespan)]
    steady = float(mid[:, 1].mean()) if len(mid) else None
    # one at a time: a measured sample, the rest modelled and calibrated on it
    g = np.random.Generator(np.random.PCG64(SEED + 11))
    pick = sorted(g.choice(len(mine), size=min(sample, len(mine)), replace=False).tolist())
    meas, model = {}, {}
    for k in pick:
        r = mine[k]
        mm = SV.build_magnets(r.spec, device=dev)
        mm.run(min(r.steps, 50))                     # warm-up: descriptors, graphs
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        mm.run(r.steps)
        e1.record()
        torch.cuda.synchronize(dev)
        meas[k] = e0.elapsed_time(e1) * 1e-3
        model[k] = modelled_alone_us(r.spec, r.steps) * 1e-6
        del mm
    calib = sum(meas.values()) / sum(model.values())
    svc = [meas[k] if k in meas else modelled_alone_us(r.spec, r.steps) * 1e-6 * calib for k, r in enumerate(mine)]
    seq_lat = SV.fifo_latencies([r.arrival for r in mine], svc)
    seq_end = max(a + l for a, l in zip([r.arrival for r in mine], seq_lat))
    mine_stats = dict(lat=[x.latency for x in res], att=sum(x.attempts for x in res), makespan=srv.stats.makespan,
                      seq_lat=list(seq_lat), seq_end=seq_end, rounds=srv.stats.rounds, max_active=srv.stats.max_active,
                      peak=srv.stats.admitted_bytes_peak, budget=srv.hbm_budget, steady=steady, calib=calib,
                      sample_s=sum(meas.values()), peak_alloc=peak_alloc, build_s=srv.stats.build_s,
                      last_active=srv.stats.last_active_s, round_ms=srv.stats.round_ms_sum,
                      sm_s=srv.stats.sm_us_sum * 1e-6, sm_s_one=srv.stats.sm_us_one_cta * 1e-6,
                      sm_s_meas=srv.stats.measured_sm_us * 1e-6, rounds_diag=rounds_diag,
                      n_sm=srv.n_sm,
                      finish_p90=float(np.percentile([x.finished for x in res], 90)))
    allst = [mine_stats]
    if dist:
        allst = [None] * ws
        dist.all_gather_object(allst, mine_stats)
    if rank != 0:
        return None
    lat = np.concatenate([np.asarray(a['lat']) for a in allst])
    seq = np.concatenate([np.asarray(a['seq_lat']) for a in allst])
    att = sum(a['att'] for a in allst)
    makespan = max(a['makespan'] for a in allst)
    seq_end = max(a['seq_end'] for a in allst)
    return {"workload": SERVED_WORKLOAD.format(k=args.served), "requests": int(lat.size),
            "placement": args.served_placement if ws > 1 else "one rank",
            "value": att / makespan, "unit": UNIT, "makespan_s": makespan, "attempts": att,
            "arrivals_span_s": float(max(r.arrival for r in reqs)),
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "rounds": sum(a['rounds'] for a in allst),
            "max_resident": max(a['max_active'] for a in allst),
            "steady_resident_mean": allst[0]['steady'],
            "hbm_budget_bytes": allst[0]['budget'], "peak_admitted_bytes": max(a['peak'] for a in allst),
            "peak_allocated_bytes": max(a['peak_alloc'] for a in allst),
            "host_build_s": sum(a['build_s'] for a in allst),
            "last_request_resident_s": max(a['last_active'] for a in allst),
            "round_device_s": sum(a['round_ms'] for a in allst) * 1e-3,
            "modelled_sm_s": sum(a['sm_s'] for a in allst),
            "modelled_sm_s_one_cta": sum(a['sm_s_one'] for a in allst),
            "measured_sm_s": sum(a['sm_s_meas'] for a in allst),
            "rounds_diag": allst[0]['rounds_diag'],
            "sm_time_note": "SM time of all quanta: planned (the step-time model scaled per request by its measured "
                            "quanta) at the planned cluster sizes, the same on one CTA each, and measured by the engine "
                            "(device time per quantum x CTAs); / (round_device_s x SMs) is the SM use of the rounds",
            "n_sm": allst[0]['n_sm'],
            "finish_p90_s": max(a['finish_p90'] for a in allst),
            "sequential": {"p50_s": float(np.percentile(seq, 50)), "p99_s": float(np.percentile(seq, 99)),
                           "makespan_s": seq_end, "value": att / seq_end,
                           "sample": f"{len(pick)} requests run alone to completion ({allst[0]['sample_s']:.1f} s of "
                                     f"device time); measured / modelled service time on them = {allst[0]['calib']:.3f}",
                           "form": "one request at a time (Magnets.run, the lone-instance engine launch), FIFO over the "
                                   "same arrivals; service times measured for the sample, modelled x the sample's "
                                   "calibration for the rest"},
            "served_over_sequential": seq_end / makespan,
            "latency_clock": "host wall clock from each request's arrival to its result on the host"}


def _counters_dtype():
    from hotspice_b200 import _lib
    return _lib.COUNTERS_DTYPE


C1_WORKLOAD = ("OOP_Square 64x64 (4096 magnets), a=200nm, moment=1.1e-15, E_B=5e-20 J uniform, T=300K, DipolarEnergy "
               "with the full untruncated kernel, iid +-1 start (p=0.5, seeded), Neel-Arrhenius single switches, "
               "{steps} steps (FP32 increments into FP64 energies, FP64 simulated time)")


def run_c1(dev, stream, steps=10000, cpu_seconds=5.0):
    """The c1 workload: one 64 x 64 OOP square lattice with the full dipolar kernel, `steps`
    Néel steps through Magnets.run on its autotuned single-instance path, timed with CUDA
    events; beside it the NumPy oracle on the same lattice for a bounded sample of steps."""
    import torch
    import hotspice_b200 as hs
    from hotspice_b200.engine import Autotuner
    from oracle.geometry import oop_square
    from oracle.hotspice_oracle import OracleDipolar, OracleMagnets
    g = np.random.Generator(np.random.PCG64(SEED + 11))
    m0 = g.integers(0, 2, size=(64, 64)) * 2 - 1
    mm = hs.ASI.OOP_Square(200e-9, 64, T=300.0, E_B=5e-20, moment=1.1e-15, pattern=m0, energies=[hs.DipolarEnergy()],
                           seed=SEED + 11, device=dev)
    choice = Autotuner().tune(mm, steps=200, include_step_kernels=True)
    mm.run(1000)
    torch.cuda.synchronize(dev)
    a0, s0 = mm.attempted_switches, mm.switches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    mm.run(steps)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1)
    att = mm.attempted_switches - a0
    mo = OracleMagnets(oop_square(200e-9, 64), m0, T=300.0, E_B=5e-20, moment=1.1e-15, energies=[OracleDipolar()],
                       seed=SEED + 11)
    mo.update()
    k, t0 = 0, time.perf_counter()
    while k < steps and time.perf_counter() - t0 < cpu_seconds:
        mo.update()
        k += 1
    cpu_s = time.perf_counter() - t0
    return {"workload": C1_WORKLOAD.format(steps=steps), "steps": steps, "ms": ms, "us_per_step": ms * 1e3 / steps,
            "value": att / (ms * 1e-3), "unit": UNIT, "switches": int(mm.switches - s0),
            "path": "per-step kernels (CUDA graphs)" if choice == 0 else f"engine cluster {choice}",
            "cpu_baseline": {"value": k / cpu_s, "unit": UNIT, "cores": 1, "kind": "port",
                             "sample": f"{k} Neel steps of the same lattice with the NumPy oracle ({cpu_s:.1f} s)"},
            "gpu_over_cpu": (att / (ms * 1e-3)) / (k / cpu_s)}


def run_single(dev, stream):
    """The 512 x 512 pinwheel instance, best single-instance path chosen by measurement."""
    import torch
    from hotspice_b200.engine import Autotuner
    mm = build_single(dev)
    r = 20 * A1
    choice = Autotuner().tune(mm, steps=200, r=r, include_step_kernels=True)
    for _ in range(2):
        mm.run(1000, r=r)
    torch.cuda.synchronize(dev)
    a0 = mm.attempted_switches
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(3):
        mm.run(1000, r=r)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1)
    att = mm.attempted_switches - a0
    return {"workload": WORKLOAD1, "value": att / (ms * 1e-3), "unit": UNIT, "us_per_mc_step": ms * 1e3 / 3000,
            "path": "per-step kernels (CUDA graphs)" if choice == 0 else f"engine cluster {choice}"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=10)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='product', choices=['product', 'reference'])
    ap.add_argument('--instances', type=int, default=N_INST)
    ap.add_argument('--mc-steps', type=int, default=STEPS_PER_BENCH_STEP, help='update steps per instance per bench step')
    ap.add_argument('--plain-sample', type=int, default=8)
    ap.add_argument('--plain-steps', type=int, default=100)
    ap.add_argument('--no-plain-best', dest='plain_best', action='store_false',
                    help='skip the best single-instance form (Magnets.run per instance, autotuned)')
    ap.add_argument('--ref-steps', type=int, default=2, help='steps of every instance per reference-arm bench step')
    ap.add_argument('--cpu-seconds', type=float, default=2.5)
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-single', action='store_true')
    ap.add_argument('--served', type=int, default=2000, help='requests of the served arrival stream (0: skip)')
    ap.add_argument('--only-served', action='store_true', help='run only the served stream and print it')
    ap.add_argument('--served-placement', default='static', choices=['static', 'dynamic'],
                    help='with several ranks: a fixed split of the stream by estimated work (static), or '
                         'requests claimed at run time by the least-loaded rank (dynamic)')
    ap.add_argument('--recompute-n', type=int, default=2048, help='lattice side of the full-recompute timing (0: skip)')
    ap.add_argument('--only-recompute', action='store_true', help='run only the full-recompute timing and print it')
    ap.add_argument('--incremental-n', type=int, default=2048, help='lattice side of the incremental-update timing (0: skip)')
    ap.add_argument('--only-incremental', action='store_true', help='run only the incremental-update timing and print it')
    ap.add_argument('--relax-n', type=int, default=1024, help='lattice side of the relax() timing (0: skip)')
    ap.add_argument('--only-relax', action='store_true', help='run only the relax() timing and print it')
    ap.add_argument('--reservoir-n', type=int, default=256, help='lattice side of the reservoir I/O timing (0: skip)')
    ap.add_argument('--only-reservoir', action='store_true', help='run only the reservoir I/O timing and print it')
    ap.add_argument('--c3-n', type=int, default=2048, help='lattice side of the Poisson-disc / resync workload')
    ap.add_argument('--c3-steps', type=int, default=5000, help='steps per temperature of that workload (0: skip)')
    ap.add_argument('--only-c3', action='store_true', help='run only the Poisson-disc / resync workload and print it')
    ap.add_argument('--c1-steps', type=int, default=10000, help='Neel steps of the 64x64 full-kernel workload (0: skip)')
    ap.add_argument('--only-c1', action='store_true', help='run only the 64x64 full-kernel Neel workload and print it')
    args = ap.parse_args()
    if args.impl == 'reference':
        run_reference(args)
    elif args.only_incremental:
        import torch
        dev = torch.device('cuda', 0)
        torch.cuda.set_device(dev)
        print(json.dumps({"incremental_update": run_incremental(dev, n=args.incremental_n)}))
    elif args.only_reservoir:
        import torch
        dev = torch.device('cuda', 0)
        torch.cuda.set_device(dev)
        print(json.dumps({"reservoir": run_reservoir(dev, n=args.reservoir_n)}))
    elif args.only_relax:
        import torch
        dev = torch.device('cuda', 0)
        torch.cuda.set_device(dev)
        print(json.dumps({"relax": run_relax(dev, n=args.relax_n)}))
    elif args.only_served:
        import torch
        dev = torch.device('cuda', 0)
        torch.cuda.set_device(dev)
        print(json.dumps({"served": run_served(dev, args, None, 0, 1)}))
    elif args.only_c1:
        import torch
        dev = torch.device('cuda', 0)
        torch.cuda.set_device(dev)
        print(json.dumps({"c1_neel": run_c1(dev, torch.cuda.current_stream(dev), steps=args.c1_steps)}))
    elif args.only_c3:
        import torch
        dev = torch.device('cuda', 0)
        torch.cuda.set_device(dev)
        print(json.dumps({"c3_poisson_resync": run_c3(dev, n=args.c3_n, steps=args.c3_steps)}))
    elif args.only_recompute:
        import torch
        dev = torch.device('cuda', 0)
        torch.cuda.set_device(dev)
        print(json.dumps({"full_recompute": run_recompute(dev, n=args.recompute_n)}))
    else:
        run_product(args)


if __name__ == '__main__':
    main()
