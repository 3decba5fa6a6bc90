"""Parity at the sizes of the benchmark configurations (seeded synthetic lattices).

c1: OOP square 64 x 64 (4096 magnets), a = 200 nm, moment 1.1e-15 A m^2, E_B = 5e-20 J, T = 300 K,
    DipolarEnergy with the full uncut kernel, iid +-1 start, Néel-Arrhenius, 10,000 steps, in
    lock-step with the FP64 oracle (hotspice/core.py:679-709, energies.py:310-329).
c2: IP pinwheel 512 x 512 (131,072 magnets), a = 300 nm, moment 1e-15, E_B lognormal (mean
    6e-20 J, 5 %), T = 300 K, DipolarEnergy cut off at 20a plus ZeemanEnergy 1 mT at 22.5 deg,
    Metropolis with grid multisampling at r = 20a, 1,000 steps, FP32 increments against the FP64
    oracle in lock-step (core.py:659-677, energies.py:331-366), and against an FP64 recompute.
c3: OOP square 2048 x 2048 (4.19 M magnets), full kernel: the tensor-core implicit GEMM
    recompute against the FP64 direct sum over every pair (energies.py:290-308).

Tolerances: energies 2e-6 relative to max |E| after the run (1e-6 right after a recompute);
near-threshold decisions at most 1 % of the decisions (tests/lockstep.py); simulated time
within the bound derived step by step from the energy differences (tests/lockstep.py).
"""
import math

import numpy as np
import pytest

from cases import build_oracle, rel_err
from gpu_cases import build_product
from lockstep import E_TOL, assert_time_within, near_bound, run_metropolis, run_neel

pytestmark = pytest.mark.gpu


def _np(t):
    return t.detach().cpu().numpy()


def c1_case(seed=20261204):
    n, a = 64, 200e-9
    g = np.random.Generator(np.random.PCG64(seed))
    spec = {'lattice': 'OOP_Square', 'a': a, 'moment': 1.1e-15, 'nx': n, 'ny': n, 'seed': seed,
            'energies': [{'type': 'dipolar'}]}
    fx = {'T': 300.0, 'E_B': np.full((n, n), 5e-20), 'm0': g.integers(0, 2, size=(n, n)) * 2 - 1}
    return spec, fx


def c2_case(seed=20261205):
    n, a = 512, 300e-9
    g = np.random.Generator(np.random.PCG64(seed))
    spec = {'lattice': 'IP_Pinwheel', 'a': a, 'moment': 1e-15, 'nx': n, 'ny': n, 'seed': seed,
            'energies': [{'type': 'dipolar', 'cutoff': 20 * a}, {'type': 'zeeman', 'B': 1e-3, 'angle': math.radians(22.5)}],
            'params': {'UPDATE_SCHEME': 'Metropolis'}}
    fx = {'T': 300.0, 'E_B': 6e-20 * g.lognormal(-0.05 ** 2 / 2, 0.05, size=(n, n)),
          'm0': g.integers(0, 2, size=(n, n)) * 2 - 1}
    return spec, fx


def test_c1_neel_oop64_full_kernel_10k_steps():
    spec, fx = c1_case()
    mo = build_oracle('c1', spec=spec, fx=fx)
    mp = build_product('c1', spec=spec, fx=fx)
    assert rel_err(_np(mp.E), mo.E) < E_TOL
    steps = 10_000
    near, decisions, t_bound = run_neel(mp, mo, steps)
    assert int(mp._read_counters()['rng_call']) == mo.rng.call
    assert mp.attempted_switches == mo.attempted_switches == steps
    assert mp.switches == mo.switches
    assert np.array_equal(_np(mp.m), mo.m)
    e = rel_err(_np(mp.E), mo.E)
    assert e < 2 * E_TOL
    err, lim = assert_time_within(mp, mo, t_bound, 'c1')
    assert near <= near_bound(decisions)
    print(f'c1: {steps} Néel steps, {mp.switches} switches, {near} near-threshold decisions, rel E err {e:.2e}, '
          f't = {mo.t:.6e}, |dt| {err:.2e} <= bound {lim:.2e}')


def test_c2_metropolis_pinwheel512_1k_steps():
    spec, fx = c2_case()
    mo = build_oracle('c2', spec=spec, fx=fx)
    mp = build_product('c2', spec=spec, fx=fx)
    assert rel_err(_np(mp.E), mo.E) < E_TOL
    kw = {'r': 20 * spec['a']}
    steps = 1000
    near, decisions, _ = run_metropolis(mp, mo, steps, kw)
    assert mp.attempted_switches == mo.attempted_switches
    assert mp.switches == mo.switches
    assert np.array_equal(_np(mp.m), mo.m)
    e = rel_err(_np(mp.E), mo.E)
    ep = rel_err(_np(mp.E_perp), mo.perp_energy())
    assert e < 2 * E_TOL and ep < 2 * E_TOL
    assert near <= near_bound(decisions)
    # the FP32 increments against an FP64 recompute of the final state (valid where the
    # kernel is symmetric: a pair exactly at the cutoff kept one way only drifts in the
    # reference algorithm too)
    d = mp._dipolar()
    E_inc = d._E.double().clone()
    d.update(method='direct64')
    e_re = float((E_inc - d._E).abs().max() / d._E.abs().max())
    if d.kernel_set.asymmetry < 1e-12:
        assert e_re < 2 * E_TOL
    print(f'c2: {steps} Metropolis steps, {decisions} candidates, {mp.switches} switches, {near} near-threshold, '
          f'rel E err vs oracle {e:.2e} (perp {ep:.2e}), vs FP64 recompute {e_re:.2e} '
          f'(kernel asymmetry {d.kernel_set.asymmetry:.1e})')


def test_c3_igemm_oop2048_against_fp64_direct():
    """Every pair of the 4.19 M-magnet lattice: the split-BF16 tensor-core GEMM (3 splits, FP32
    TMEM accumulation flushed to FP64, near field in FP64) against the FP64 direct sum."""
    import torch
    import hotspice_b200 as hs
    n = 2048
    mm = hs.ASI.OOP_Square(200e-9, n, T=300.0, E_B=5e-20, moment=1.1e-15, pattern='random', seed=33,
                           energies=[hs.DipolarEnergy()], engine=hs.EngineConfig(recompute='igemm'))
    d = mm._dipolar()
    d.update(method='igemm')
    E_ig = d._E.clone()
    d.update(method='direct64')
    torch.cuda.synchronize()
    E64 = d._E
    err = float((E_ig - E64).abs().max() / E64.abs().max())
    etot = abs(float(E_ig.sum()) - float(E64.sum())) / abs(float(E64.sum()))
    print(f'c3: igemm vs FP64 direct at {n}^2: max rel err {err:.2e}, E_tot rel err {etot:.2e}')
    assert err <= E_TOL
    assert etot <= E_TOL
