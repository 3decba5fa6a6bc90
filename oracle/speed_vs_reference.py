"""Times the unmodified reference (hotspice, NumPy path) against the oracle on instances of the
benchmark batch, one NumPy thread each, so that a rate measured with the oracle can be read as
the reference's own. Test infrastructure: it needs the reference checkout, so it runs only where
that exists:

    python oracle/speed_vs_reference.py --ref <reference checkout> [--every 16] [--steps 5]

The reference is loaded as tests/golden/make_golden.py does (its hotspice package without the
GUI and plotting modules, three display-only imports stubbed) and its random draws are routed
through the oracle's Philox stream; both sides build the same lattice, energies, start state and
E_B of each instance and step it `steps` times. Prints one JSON line per instance and a summary.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, 'tests', 'golden'))

for _v in ('OMP_NUM_THREADS', 'OPENBLAS_NUM_THREADS', 'MKL_NUM_THREADS'):
    os.environ[_v] = '1'

import numpy as np  # noqa: E402


def reference_instance(hs, spec):
    import bench
    m0, EB = bench.instance_inputs(spec)
    cls = getattr(hs.ASI, spec['lattice'])
    mm = cls(spec['a'], spec['n'], T=spec['T'], E_B=EB, moment=spec['moment'],
             energies=[hs.energies.DipolarEnergy(cutoff_range=16 * spec['a']),
                       hs.energies.ZeemanEnergy(spec['B'], spec['angle'])],
             params=hs.core.SimParams(UPDATE_SCHEME=spec['scheme']))
    mm.initialize_m(m0 * mm.occupation)
    return mm


def timed(mm, steps):
    mm.update()                      # first step outside the timing (lazy set-up)
    t0 = time.perf_counter()
    a0 = mm.attempted_switches
    for _ in range(steps):
        mm.update()
    return time.perf_counter() - t0, mm.attempted_switches - a0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--ref', default=os.environ.get('HOTSPICE_REFERENCE'), help='reference checkout')
    ap.add_argument('--every', type=int, default=16, help='time every k-th instance of the batch')
    ap.add_argument('--steps', type=int, default=5)
    args = ap.parse_args()
    if not args.ref:
        ap.error('the reference checkout is required: --ref <dir> or HOTSPICE_REFERENCE=<dir>')
    import bench
    from make_golden import load_reference, route_rng
    from oracle.philox import PhiloxStream
    hs = load_reference(args.ref)
    ratios, t_ref, t_or = [], 0.0, 0.0
    for spec in bench.instance_specs()[::args.every]:
        ref = reference_instance(hs, spec)
        route_rng(ref, PhiloxStream(spec['seed']))
        ora = bench.build_oracle_instance(spec)
        sr, ar = timed(ref, args.steps)
        so, ao = timed(ora, args.steps)
        ratios.append(sr / so)
        t_ref += sr
        t_or += so
        print(json.dumps({'i': spec['i'], 'lattice': spec['lattice'], 'n': spec['n'], 'scheme': spec['scheme'],
                          'reference_ms_per_step': 1e3 * sr / args.steps, 'oracle_ms_per_step': 1e3 * so / args.steps,
                          'reference_over_oracle_time': sr / so, 'attempts': [int(ar), int(ao)]}), flush=True)
    print(json.dumps({'instances': len(ratios), 'steps_each': args.steps,
                      'total_time_reference_over_oracle': t_ref / t_or,
                      'median_ratio': float(np.median(ratios)), 'min_ratio': float(min(ratios)),
                      'max_ratio': float(max(ratios))}))


if __name__ == '__main__':
    main()
