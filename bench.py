"""Benchmark of the kinetic Monte Carlo hot path on B200.

Workload (one bench step): the in-plane pinwheel lattice of 512 x 512 cells (131,072
magnets, a = 300 nm, moment 1e-15 A m^2, E_B lognormal with mean 6e-20 J and 5 % sigma,
T = 300 K), dipolar interaction cut off at 20a plus a 1 mT Zeeman field at 22.5 degrees,
advanced by 1,000 Metropolis multisample steps with the grid selection at spacing r = 20a,
FP32 incremental energy updates. Seeded synthetic inputs (no dataset is involved).

  value : switch-attempts/s with the state resident in HBM (steps replayed from captured
          CUDA graphs, no host synchronisation inside a bench step), L2 flushed between
          bench steps.
  e2e   : the same metric through the public API (Magnets.progress) with the start state
          copied in from pinned host memory and the final spins and counters copied out,
          every bench step.

Multi-GPU: one independent lattice per rank (the work shards into independent instances,
no data-path collective); value = all ranks' attempts / max-over-ranks device time.

`--impl reference` times the reference algorithm's NumPy restatement (the oracle) on the host
cores on a bounded sample of the same workload.
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
A = 300e-9
N = 512
STEPS_PER_BENCH_STEP = 1000
SEED = 20261203
WORKLOAD = ("IP_Pinwheel 512x512 (131072 magnets), a=300nm, moment=1e-15, E_B lognormal(6e-20, 5%), T=300K, "
            "dipolar cutoff 20a + Zeeman 1mT@22.5deg, Metropolis grid r=20a, 1000 multisample steps per bench step, FP32")


def workload_inputs(seed=SEED):
    g = np.random.Generator(np.random.PCG64(seed))
    m0 = g.integers(0, 2, size=(N, N)) * 2 - 1
    EB = 6e-20 * g.lognormal(-0.05 ** 2 / 2, 0.05, size=(N, N))
    return m0, EB


def build_product(device, seed=SEED):
    import hotspice_b200 as hs
    m0, EB = workload_inputs(seed)
    mm = hs.ASI.IP_Pinwheel(A, N, T=300.0, E_B=EB, moment=1e-15, pattern=m0,
                            energies=[hs.DipolarEnergy(cutoff_range=20 * A),
                                      hs.ZeemanEnergy(1e-3, math.radians(22.5))],
                            params=hs.SimParams(UPDATE_SCHEME='Metropolis', MULTISAMPLING_SCHEME='grid'),
                            seed=seed, device=device,
                            engine=hs.EngineConfig(graph_steps=100))
    return mm


def build_oracle(seed=SEED):
    from oracle.geometry import ip_pinwheel
    from oracle.hotspice_oracle import OracleDipolar, OracleMagnets, OracleZeeman
    m0, EB = workload_inputs(seed)
    return OracleMagnets(ip_pinwheel(A, N), m0, T=300.0, E_B=EB, moment=1e-15,
                         energies=[OracleDipolar(cutoff_range=20 * A), OracleZeeman(1e-3, math.radians(22.5))],
                         params=dict(UPDATE_SCHEME='Metropolis'), seed=seed)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""
    Q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,'
         'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,'
         'clocks_event_reasons.sw_power_cap')

    def __init__(self, index):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(['nvidia-smi', f'--query-gpu={self.Q}', '--format=csv,noheader,nounits',
                                      '-i', str(self.index)], capture_output=True, text=True, timeout=5).stdout
                self.rows.append([c.strip() for c in out.strip().split(',')])
            except Exception:
                pass
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
        import torch.distributed as dist
        import datetime
        backend = 'nccl'
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
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
    """Per-launch DRAM traffic of the update kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, 'profiles', 'engine_kernel_pinwheel512.txt')
    try:
        for line in open(path):
            if line.startswith('traffic_bytes_per_launch:'):
                return float(line.split(':', 1)[1])
    except OSError:
        pass
    return None


def cpu_baseline_sample(steps=60):
    """The oracle (NumPy restatement of the reference) on a bounded sample of the workload."""
    mo = build_oracle()
    r = 20 * A
    for _ in range(3):
        mo.update(r=r)
    a0 = mo.attempted_switches
    t0 = time.perf_counter()
    for _ in range(steps):
        mo.update(r=r)
    dt = time.perf_counter() - t0
    return (mo.attempted_switches - a0) / dt, dt, steps


def run_reference(args):
    rank, ws = int(os.environ.get('RANK', '0')), int(os.environ.get('WORLD_SIZE', '1'))
    if rank != 0:
        return
    mo = build_oracle()
    r = 20 * A
    sample = args.ref_sample
    for _ in range(args.warmup):
        for _ in range(sample):
            mo.update(r=r)
    att, secs = 0, 0.0
    for _ in range(args.steps):
        a0 = mo.attempted_switches
        t0 = time.perf_counter()
        for _ in range(sample):
            mo.update(r=r)
        secs += time.perf_counter() - t0
        att += mo.attempted_switches - a0
    v = att / secs
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample_steps_per_bench_step": sample},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
                             "sample": f"{sample} Metropolis steps per bench step of the 512x512 workload "
                                       f"(NumPy oracle restating the reference, single process)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_product(args):
    import torch
    dist, rank, ws, local = dist_setup()
    dev = torch.device('cuda', local)
    torch.cuda.set_device(dev)
    from hotspice_b200.engine import Autotuner
    mcs = args.mc_steps
    mm = build_product(dev, seed=SEED + rank)
    r = 20 * A
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    d = mm.get_energy('dipolar')
    cs = Autotuner().tune(mm, steps=200, r=r) if not args.cluster_size else args.cluster_size
    mm.engine.cluster_size = cs

    # pinned host copies of the start state for the end-to-end leg
    snap = {k: v.detach().clone() for k, v in (('m', mm._m_dev), ('mm', mm._mm_dev), ('E', d._E), ('Ep', d._Ep),
                                               ('C', mm._counters))}
    host_in = {k: v.cpu().pin_memory() for k, v in snap.items()}
    host_out_m = torch.empty_like(mm._m_dev, device='cpu').pin_memory()
    host_out_c = torch.empty_like(mm._counters, device='cpu').pin_memory()
    h2d = sum(v.numel() * v.element_size() for v in host_in.values())
    d2h = host_out_m.numel() + host_out_c.numel()

    # ---- device-resident throughput: one persistent launch per bench step ----------------
    for _ in range(args.warmup):
        mm.run(mcs, r=r)
    torch.cuda.synchronize(dev)
    c0 = mm._read_counters()
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    sampler = ClockSampler(local)
    with sampler:
        for k in range(args.steps):
            flush.fill_(float(k))
            ev[k][0].record(stream)
            mm.run(mcs, r=r)
            ev[k][1].record(stream)
        torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    dev_ms = sum(a.elapsed_time(b) for a, b in ev)
    c1 = mm._read_counters()
    attempts = int(c1['attempted'] - c0['attempted'])
    switches = int(c1['switches'] - c0['switches'])
    status = int(c1['status'])

    # ---- roofline of the fused engine kernel (the only kernel of a bench step) ------------
    ks = d.kernel_set
    W = (2 * ks.wx + 1) * (2 * ks.wy + 1)
    # per switch: E f32 read+write, kernel, source m*mu (16 B) and E_perp read+write, perp kernel
    # (12 B) for every window cell; per candidate: E, E_perp, Zeeman factor, beta-free E_B, spin
    alg_bytes = (switches * W * 28 + attempts * 17) / args.steps
    launch_ms = dev_ms / args.steps
    hbm, peak_kind = measured_peaks()
    achieved = alg_bytes / (launch_ms * 1e-3) / 1e9

    # ---- end to end through the public API ------------------------------------------------
    mc_per_step = attempts / max(args.steps, 1) / mm.n
    for _ in range(max(1, args.warmup // 2)):
        mm.progress(t_max=math.inf, MCsteps_max=mc_per_step, r=r)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    e2e_att = 0
    t_e2e = time.perf_counter()
    ee0, ee1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ee0.record(stream)
    for k in range(args.steps):
        mm._m_dev.copy_(host_in['m'], non_blocking=True)
        mm._mm_dev.copy_(host_in['mm'], non_blocking=True)
        d._E.copy_(host_in['E'], non_blocking=True)
        d._Ep.copy_(host_in['Ep'], non_blocking=True)
        mm._counters.copy_(host_in['C'], non_blocking=True)
        mm._ctl = None
        dt_, dmc = mm.progress(t_max=math.inf, MCsteps_max=mc_per_step, r=r)
        e2e_att += int(round(dmc * mm.n))
        host_out_m.copy_(mm._m_dev, non_blocking=True)
        host_out_c.copy_(mm._counters, non_blocking=True)
    ee1.record(stream)
    torch.cuda.synchronize(dev)
    e2e_ms = ee0.elapsed_time(ee1)
    wall_e2e = time.perf_counter() - t_e2e

    # ---- reductions over ranks -------------------------------------------------------------
    vals = torch.tensor([dev_ms, e2e_ms, float(attempts), float(e2e_att)], dtype=torch.float64, device=dev)
    if dist:
        mx = vals.clone(); dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        sm = vals.clone(); dist.all_reduce(sm, op=dist.ReduceOp.SUM)
        dev_ms, e2e_ms = float(mx[0]), float(mx[1])
        attempts, e2e_att = int(sm[2]), int(sm[3])
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    value = attempts / (dev_ms * 1e-3)
    e2e_value = e2e_att / (e2e_ms * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": dev_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded lattice, random start, lognormal E_B)",
        "config": {"workload": WORKLOAD, "lattice": "IP_Pinwheel", "nx": N, "ny": N, "magnets": mm.n,
                   "steps_per_bench_step": mcs, "l2": "flushed (256 MB write) between bench steps",
                   "parallelism": f"{ws} independent replicas" if ws > 1 else "single instance",
                   "cluster_size": cs, "switches": switches, "attempts": attempts, "device_status": status},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "api": "Magnets.progress(t_max=inf, MCsteps_max=per-step share) with state restored from pinned host",
                "wall_s": wall_e2e},
        "gpu_launches": launches_for(args.steps),
        "roofline": {"bound": "hbm", "kernel": f"engine_kernel<{cs}>", "achieved": achieved, "peak": hbm,
                     "unit": "GB/s", "frac": achieved / hbm, "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                     "traffic": profile_traffic(), "launch_ms": launch_ms,
                     "algorithmic_bytes_per_launch": alg_bytes, "window_cells": W},
        "clocks": sampler.summary(),
    }
    if not args.no_cpu_baseline:
        v, secs, st = cpu_baseline_sample(args.cpu_steps)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
                                "sample": f"{st} Metropolis steps of the same 512x512 workload ({secs:.1f} s) with the "
                                          f"NumPy oracle restating the reference"}
    print(json.dumps(line))
    if dist:
        dist.destroy_process_group()


def launches_for(steps):
    return steps  # one persistent engine launch per bench step


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=10)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='product', choices=['product', 'reference'])
    ap.add_argument('--ref-sample', type=int, default=40)
    ap.add_argument('--cpu-steps', type=int, default=400)
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--mc-steps', type=int, default=STEPS_PER_BENCH_STEP,
                    help='Metropolis steps per bench step (the workload uses 1000)')
    ap.add_argument('--cluster-size', type=int, default=0, help='CTAs per cluster (0: autotune)')
    args = ap.parse_args()
    if args.impl == 'reference':
        run_reference(args)
    else:
        run_product(args)


if __name__ == '__main__':
    main()
