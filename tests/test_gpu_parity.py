"""Parity of the CUDA path with the FP64 oracle (which is pinned to the reference).

Tolerances (stated by the build's precision design):
* energies: the device keeps E in FP32; max|E_gpu - E_oracle| / max|E_oracle| <= 2e-6 after the
  run (<= 1e-6 right after a full recompute);
* decisions: every Néel argmin / Metropolis acceptance / Wolff bond must equal the oracle's,
  except where the decision margin is below the effect of a 1e-6 relative energy error
  ("near-threshold"); those are counted (at most 1% of the decisions, plus one), the oracle is
  then forced to the device's decision so both continue in lock-step (tests/lockstep.py);
* simulated time: within the bound derived step by step from the energy difference before
  each step (tests/lockstep.py states it);
* Wolff clusters are integer decisions against FP64 thresholds: exact, no exceptions.
"""
import numpy as np
import pytest

from cases import build_oracle, dipolar_like, load_fixture, load_specs, rel_err
from gpu_cases import build_product
from lockstep import E_TOL, assert_time_within, near_bound, run_metropolis, run_neel, run_progress

pytestmark = pytest.mark.gpu
SPECS = load_specs()


def _np(t):
    return t.detach().cpu().numpy()


def _scheme(spec):
    return spec.get('params', {}).get('UPDATE_SCHEME', 'Neel')


def test_philox_device_matches_numpy():
    import torch
    from hotspice_b200 import _lib
    from oracle.philox import uniform53
    lib = _lib.load()
    for seed, call, n in ((0, 0, 1000), (2 ** 64 - 1, 12345, 4097), (77, 2 ** 40 + 3, 33)):
        out = torch.empty(n, dtype=torch.float64, device='cuda')
        _lib.check(lib.hs_philox_uniform(seed, call, n, out.data_ptr(), torch.cuda.current_stream().cuda_stream))
        assert np.array_equal(_np(out), uniform53(seed, call, n))


@pytest.mark.parametrize('name', [n for n in SPECS if any(e['type'] in ('dipolar', 'dimonopolar') for e in SPECS[n]['energies'])])
def test_full_recompute_matches_oracle(name):
    fx = load_fixture(name)
    mp = build_product(name)
    d = dipolar_like(mp)
    assert rel_err(_np(d.E), fx['E_dip_init']) < 1e-6
    if mp.USE_PERP_ENERGY:
        assert rel_err(_np(d.E_perp), fx['E_dip_perp_init']) < 1e-6
    assert rel_err(_np(mp.E), fx['E_init']) < 1e-6
    # single-precision accumulation of every (cell, kernel) product: cancellation between
    # thousands of terms costs about one decimal digit
    d.update(method='direct32')
    assert rel_err(_np(d.E), fx['E_dip_init']) < 1e-5


def _check_perp(mp, mo):
    """The magnetostatic E_perp after the run (its sign at switched magnets differs between
    DipolarEnergy and DiMonopolarEnergy multi-switch updates)."""
    dp, do = dipolar_like(mp), dipolar_like(mo)
    if dp is not None and mp.USE_PERP_ENERGY:
        assert rel_err(_np(dp.E_perp), do.E_perp) < 2 * E_TOL


@pytest.mark.parametrize('name', [n for n in SPECS if _scheme(SPECS[n]) in ('Neel',) and SPECS[n].get('steps')])
def test_neel_lockstep(name):
    spec = SPECS[name]
    mo = build_oracle(name)
    mp = build_product(name)
    near, decisions, t_bound = run_neel(mp, mo, spec['steps'])
    c = mp._read_counters()
    assert int(c['rng_call']) == mo.rng.call
    assert mp.attempted_switches == mo.attempted_switches
    assert mp.switches == mo.switches
    assert np.array_equal(_np(mp.m), mo.m)
    assert rel_err(_np(mp.E), mo.E) < 2 * E_TOL
    _check_perp(mp, mo)
    err, lim = assert_time_within(mp, mo, t_bound, name)
    assert near <= near_bound(decisions), f'{near} near-threshold decisions of {decisions}'
    print(f'{name}: {decisions} steps, {near} near-threshold decisions, |dt| {err:.2e} <= bound {lim:.2e}')


@pytest.mark.parametrize('name', [n for n in SPECS if _scheme(SPECS[n]) == 'Metropolis' and SPECS[n].get('steps')])
def test_metropolis_lockstep(name):
    spec = SPECS[name]
    kw = spec.get('update_kw', {})
    mo = build_oracle(name)
    mp = build_product(name)
    near, decisions, t_bound = run_metropolis(mp, mo, spec['steps'], kw)
    assert mp.attempted_switches == mo.attempted_switches
    assert mp.switches == mo.switches
    assert np.array_equal(_np(mp.m), mo.m)
    assert rel_err(_np(mp.E), mo.E) < 2 * E_TOL
    _check_perp(mp, mo)
    msg = ''
    if spec.get('params', {}).get('METROPOLIS_TIME'):
        err, lim = assert_time_within(mp, mo, t_bound, name)
        msg = f', |dt| {err:.2e} <= bound {lim:.2e}'
    assert near <= near_bound(decisions), f'{near} near-threshold acceptances of {decisions}'
    print(f'{name}: {spec["steps"]} steps, {decisions} candidates, {near} near-threshold acceptances{msg}')


@pytest.mark.parametrize('name', [n for n in SPECS if _scheme(SPECS[n]) == 'Wolff'])
def test_wolff_matches_reference_exactly(name):
    """Integer cluster growth: identical clusters to the reference run, step by step."""
    spec, fx = SPECS[name], load_fixture(name)
    mp = build_product(name)
    ys, xs = [], []
    for s in range(spec['steps']):
        c = mp.update()
        ys += c[0].tolist(); xs += c[1].tolist()
        assert mp.attempted_switches == fx['attempted'][s]
        assert int(mp._read_counters()['rng_call']) == fx['calls'][s]
    assert np.array_equal(ys, fx['sw_y']) and np.array_equal(xs, fx['sw_x'])
    assert np.array_equal(_np(mp.m), fx['m_final'])
    assert rel_err(_np(mp.E), fx['E_final']) < 1e-6


@pytest.mark.parametrize('name', [n for n in SPECS if SPECS[n].get('progress')])
def test_progress_matches_reference(name):
    """progress() on the device (graph-replayed chunks, stop rule evaluated by the kernels)
    against the reference run. Its time is held to a bound derived from a lock-step run of
    the same progress() with the oracle (the oracle reproduces the reference's time to 1e-9)."""
    spec, fx = SPECS[name], load_fixture(name)
    mp = build_product(name)
    dt, dmc = mp.progress(**spec['progress'])
    assert dmc == pytest.approx(fx['progress'][1], rel=1e-12)
    assert int(mp._read_counters()['rng_call']) == int(fx['progress_calls'])
    assert np.array_equal(_np(mp.m), fx['m_final'])
    assert rel_err(_np(mp.E), fx['E_final']) < 2 * E_TOL
    mb, mo = build_product(name), build_oracle(name)
    near, decisions, t_bound = run_progress(mb, mo, **spec['progress'])
    assert np.array_equal(_np(mb.m), fx['m_final'])
    assert near <= near_bound(decisions)
    lim = t_bound + 1e-9 * abs(fx['progress'][0]) + 1e-300
    assert abs(dt - fx['progress'][0]) <= lim, f'|dt - reference| {abs(dt - fx["progress"][0]):.3e} > bound {lim:.3e}'
    print(f'{name}: {decisions} decisions, {near} near-threshold, |dt - ref| {abs(dt - fx["progress"][0]):.2e} '
          f'<= {lim:.2e}')


def test_progress_graph_equals_plain_launches():
    """The graph-replayed device loop and plain per-step launches give identical states."""
    import hotspice_b200 as hs
    name = 'progress_pin16_metro'
    spec = SPECS[name]
    a = build_product(name, engine=hs.EngineConfig(persistent=False, use_graphs=True, graph_steps=8))
    b = build_product(name, engine=hs.EngineConfig(persistent=False, use_graphs=False, graph_steps=8))
    ra = a.progress(**spec['progress'])
    rb = b.progress(**spec['progress'])
    assert ra == rb
    assert np.array_equal(_np(a.m), _np(b.m))
    assert np.array_equal(_np(a.get_energy('dipolar')._E), _np(b.get_energy('dipolar')._E))


def test_update_single_and_multiple_match_oracle():
    """Energy plugin contract: update_single/update_multiple after flips in m."""
    name = 'metro_oop32_trunc_pbc'
    mo = build_oracle(name)
    mp = build_product(name)
    rng = np.random.default_rng(0)
    for k in (1, 5, 25, 60):
        flat = rng.choice(mo.nx * mo.ny, size=k, replace=False)
        idx = np.asarray(np.unravel_index(np.sort(flat), mo.shape))
        mo.m[idx[0], idx[1]] *= -1
        m = mo.m.copy()
        mp.m = m
        mo.update_energy(idx)
        mp.update_energy(idx)
        assert rel_err(_np(mp.E), mo.E) < E_TOL, k


def test_metropolis_poisson_lockstep_large():
    """Poisson-disc selection on a 192 x 192 periodic lattice at r = 5a (hundreds of points a
    step): the warp's parallel evaluation of each active point's tries, resolved in try order,
    gives the oracle's sequential Bridson candidates, and the same acceptances, step by step."""
    a, n = 200e-9, 192
    g = np.random.Generator(np.random.PCG64(78))
    spec = {'lattice': 'OOP_Square', 'a': a, 'moment': 1e-15, 'nx': n, 'ny': n, 'seed': 78, 'kw': {'PBC': True},
            'energies': [{'type': 'dipolar', 'cutoff': 6 * a}, {'type': 'zeeman', 'B': 1e-3, 'angle': 0.0}],
            'params': {'UPDATE_SCHEME': 'Metropolis', 'MULTISAMPLING_SCHEME': 'Poisson'}}
    fx = {'T': 300.0, 'E_B': 5e-20 * np.ones((n, n)), 'm0': g.integers(0, 2, size=(n, n)) * 2 - 1}
    mo = build_oracle('poisson_large', spec=spec, fx=fx)
    mp = build_product('poisson_large', spec=spec, fx=fx)
    near, decisions, _ = run_metropolis(mp, mo, 8, {'r': 5 * a})
    assert decisions > 8 * 300
    assert mp.attempted_switches == mo.attempted_switches
    assert mp.switches == mo.switches
    assert np.array_equal(_np(mp.m), mo.m)
    assert rel_err(_np(mp.E), mo.E) < 2 * E_TOL
    assert near <= near_bound(decisions)
    print(f'poisson 192^2: 8 steps, {decisions} candidates, {near} near-threshold')


def test_metropolis_poisson_lockstep():
    """Poisson-disc multisampling in cell units: the device's dart throwing (one warp)
    consumes the oracle's variates in the same order, so candidates, acceptances, switch
    counts and the Philox call count agree step by step; the candidates keep the disc
    distance (r + 1 in the continuous plane, minus the rounding to cell centres)."""
    from oracle.hotspice_oracle import force_metropolis, metropolis_decision
    a, n = 200e-9, 48
    g = np.random.Generator(np.random.PCG64(77))
    spec = {'lattice': 'OOP_Square', 'a': a, 'moment': 1e-15, 'nx': n, 'ny': n, 'seed': 77, 'kw': {'PBC': True},
            'energies': [{'type': 'dipolar', 'cutoff': 8 * a}, {'type': 'zeeman', 'B': 1e-3, 'angle': 0.0}],
            'params': {'UPDATE_SCHEME': 'Metropolis', 'MULTISAMPLING_SCHEME': 'Poisson'}}
    fx = {'T': 300.0, 'E_B': 5e-20 * np.ones((n, n)), 'm0': g.integers(0, 2, size=(n, n)) * 2 - 1}
    mo = build_oracle('poisson', spec=spec, fx=fx)
    mp = build_product('poisson', spec=spec, fx=fx)
    kw = {'r': 6 * a}
    near, total = 0, 0
    for s in range(40):
        idx, p, u, dt = metropolis_decision(mo, **kw)
        total += idx.shape[1]
        if idx.shape[1] > 1:
            d = np.abs(idx[:, :, None] - idx[:, None, :]).astype(float)
            d = np.minimum(d, n - d)
            d2 = (d ** 2).sum(0) + np.eye(idx.shape[1]) * 1e9
            assert np.sqrt(d2.min()) > 6 + 1 - np.sqrt(2)
        sw = mp.update(**kw)
        got = {(int(a_), int(b_)) for a_, b_ in zip(sw[0], sw[1])}
        acc_dev = np.array([(int(a_), int(b_)) in got for a_, b_ in zip(idx[0], idx[1])])
        assert len(got) == int(acc_dev.sum()), f'step {s}: device switched a cell that was not a candidate'
        diff = np.nonzero(acc_dev != (u < p))[0]
        if diff.size:
            Emax = np.max(np.abs(mo.E))
            beta = mo.beta[idx[0], idx[1]]
            band = p * beta * 2 * 2 * E_TOL * Emax * 1.01 + 1e-12
            assert np.all(np.abs(u - p)[diff] <= band[diff]), f'step {s}: acceptance differs beyond tolerance'
            near += diff.size
        force_metropolis(mo, idx, acc_dev, dt)
        assert mp._read_counters()['rng_call'] == mo.rng.call, f'step {s}: RNG call count diverged'
    assert total > 40
    assert mp.attempted_switches == mo.attempted_switches
    assert mp.switches == mo.switches
    assert np.array_equal(_np(mp.m), mo.m)
    assert rel_err(_np(mp.E), mo.E) < 2 * E_TOL
    print(f'poisson: 40 steps, {total} candidates, {near} near-threshold acceptances')
