"""Lock-step runners shared by the GPU parity tests: the CUDA path takes a step, the oracle
evaluates the same step's decision from its FP64 state and the same Philox variates, and the
two are compared before the oracle is advanced.

Decisions. Every Néel argmin and Metropolis acceptance must equal the oracle's, except where
the decision margin is below the effect of the stated energy tolerance E_TOL (1e-6 relative);
such a "near-threshold" decision is counted and the oracle is forced to the device's choice,
so both continue in lock-step. The count is bounded: at most NEAR_FRACTION of the decisions
(plus one), so a run in which many decisions fell inside the band would fail.

Simulated time. Both sides draw the same exponential variate E1 for a step; their switching
times differ only through the energy barrier b (hotspice/core.py:625-656), which moves by at
most Delta = 2 |dE| + |dE_perp| (|dE|, |dE_perp|: the largest difference between the device's
and the oracle's total and perpendicular energies before the step). A Néel switching time is
E1 exp(b beta) / nu (two-channel: E1 / (nu (exp(-b1 beta) + exp(-b2 beta)))) and a
METROPOLIS_TIME increment a sum of such terms, so the step's time differs by at most the
factor exp(beta_max Delta). The runners add up t_step (exp(beta_max Delta) - 1) over the steps;
the final |t_device - t_oracle| must stay within that sum plus 1e-12 t (FP64 rounding of the
running sums).
"""
from __future__ import annotations

import math

import numpy as np

E_TOL = 1e-6
NEAR_FRACTION = 0.01


def _np(t):
    return t.detach().cpu().numpy()


def near_bound(decisions):
    return NEAR_FRACTION * decisions + 1


def barrier_shift(mp, mo):
    """beta_max * Delta: the largest change of beta * (energy barrier) that the device's energy
    error can cause, from the current device and oracle energies."""
    dE = float(np.max(np.abs(_np(mp.E) - mo.E)))
    dEp = 0.0
    if mo.USE_PERP_ENERGY:
        dEp = float(np.max(np.abs(_np(mp.E_perp) - mo.perp_energy())))
    return float(np.max(mo.beta)) * (2 * dE + dEp)


def _near_neel(mo, keys, i_dev, i_or, beta_max):
    """Margin of choosing i_dev over the FP64 argmin i_or, against the effect of a 1e-6
    relative energy error on two cells' barriers (each barrier moves by <= 2 dE)."""
    Emax = np.max(np.abs(mo.E))
    tol = 2 * 2 * 2 * E_TOL * Emax * beta_max + 1e-9
    return keys[i_dev] - keys[i_or] <= tol


def run_neel(mp, mo, steps, t_max=1.0, track_time=True):
    """Néel steps in lock-step; returns (near-threshold decisions, decisions, time bound)."""
    from oracle.hotspice_oracle import force_neel, neel_decision
    near, t_bound = 0, 0.0
    beta_max = float(np.max(mo.beta))
    for s in range(steps):
        shift = barrier_shift(mp, mo) if track_time else 0.0
        keys, taus, bmin, af = neel_decision(mo)
        flat = int(np.argmin(keys))
        i_or = divmod(flat, mo.nx)
        with np.errstate(over='ignore'):
            time = taus[i_or] * np.exp(bmin * mo.beta[i_or]) / af
        sw_or = None if (time > t_max or np.isnan(time)) else i_or
        sw_dev = mp.update(t_max=t_max)
        if sw_dev != sw_or:
            if sw_dev is None or sw_or is None:
                # switch or not: the switching time is within the time bound of t_max
                assert track_time and abs(time / t_max - 1) <= math.expm1(shift) + 1e-12, \
                    f'step {s}: {sw_dev} vs {sw_or} (time {time:.6e}, t_max {t_max})'
            else:
                assert _near_neel(mo, keys, sw_dev, i_or, beta_max), f'step {s}: {sw_dev} vs {sw_or} not near-threshold'
            near += 1
        t0 = mo.t
        force_neel(mo, sw_dev, t_max=t_max)
        if sw_dev is not None:
            t_bound += (mo.t - t0) * math.expm1(shift)
    return near, steps, t_bound


def run_metropolis(mp, mo, steps, kw, track_time=None):
    """Metropolis steps in lock-step; returns (near-threshold acceptances, candidates, time
    bound). Also checks each step's candidates and Philox call count."""
    from oracle.hotspice_oracle import force_metropolis, metropolis_decision
    if track_time is None:
        track_time = bool(mo.params['METROPOLIS_TIME'])
    near, total, t_bound = 0, 0, 0.0
    for s in range(steps):
        shift = barrier_shift(mp, mo) if track_time else 0.0
        idx, p, u, dt = metropolis_decision(mo, **kw)
        total += idx.shape[1]
        acc_or = u < p
        sw = mp.update(**kw)
        got = {(int(a), int(b)) for a, b in zip(sw[0], sw[1])}
        acc_dev = np.array([(int(a), int(b)) in got for a, b in zip(idx[0], idx[1])])
        assert len(got) == int(acc_dev.sum()), f'step {s}: device switched a cell that was not a candidate'
        diff = np.nonzero(acc_dev != acc_or)[0]
        if diff.size:
            Emax = np.max(np.abs(mo.E))
            beta = mo.beta[idx[0], idx[1]]
            band = p * beta * 2 * 2 * E_TOL * Emax * 1.01 + 1e-12
            assert np.all(np.abs(u - p)[diff] <= band[diff]), f'step {s}: acceptance differs beyond tolerance'
            near += diff.size
        force_metropolis(mo, idx, acc_dev, dt)
        t_bound += dt * math.expm1(shift)
        assert mp._read_counters()['rng_call'] == mo.rng.call, f'step {s}: RNG call count diverged'
    return near, total, t_bound


def assert_time_within(mp, mo, t_bound, what=''):
    if math.isinf(mo.t) or math.isinf(mp.t):
        # a step time overflowed to +inf (exp of a huge barrier), in the reference too: both must
        assert mp.t == mo.t, f'{what}: t_dev = {mp.t}, t_oracle = {mo.t}'
        return 0.0, 0.0
    err = abs(mp.t - mo.t)
    lim = t_bound + 1e-12 * abs(mo.t) + 1e-300
    assert err <= lim, f'{what}: |t_dev - t_oracle| = {err:.3e} > derived bound {lim:.3e} (t = {mo.t:.6e})'
    return err, lim


def run_progress(mp, mo, t_max=1.0, MCsteps_max=4.0, **kw):
    """progress(t_max, MCsteps_max) (hotspice/core.py:736-760) in lock-step: the oracle's stop
    rule, each Néel step bounded by the remaining time; returns (near, decisions, time bound)."""
    from oracle.hotspice_oracle import lower_than
    t0, mc0 = mo.t, mo.MCsteps
    near = dec = 0
    t_bound = 0.0
    neel = mo.params['UPDATE_SCHEME'] in ('Neel', 'Néel')
    while lower_than(mo.t - t0, t_max) and lower_than(mo.MCsteps - mc0, MCsteps_max):
        if neel:
            n, d, b = run_neel(mp, mo, 1, t_max=t_max - (mo.t - t0))
        else:
            n, d, b = run_metropolis(mp, mo, 1, kw, track_time=True)
        near, dec, t_bound = near + n, dec + d, t_bound + b
    return near, dec, t_bound
