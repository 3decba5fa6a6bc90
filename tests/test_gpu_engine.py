"""Persistent cluster engine: identical results to the per-step kernels, for every cluster
size, and identical results for an instance run alone or inside a mixed batch."""
import numpy as np
import pytest

from cases import dipolar_like, load_specs
from gpu_cases import build_product

pytestmark = pytest.mark.gpu
SPECS = load_specs()


def _state(mm):
    d = dipolar_like(mm)
    c = mm._read_counters()
    return (mm._m_dev.cpu().numpy(), None if d is None else d._E.cpu().numpy(),
            None if d is None or d._Ep is None else d._Ep.cpu().numpy(),
            {k: c[k] for k in ('attempted', 'switches', 'rng_call', 't', 'status')})


def _assert_same(a, b, what):
    assert np.array_equal(a[0], b[0]), f'{what}: spins differ'
    for i in (1, 2):
        if a[i] is not None:
            assert np.array_equal(a[i], b[i]), f'{what}: energies differ (max {np.max(np.abs(a[i] - b[i]))})'
    assert a[3] == b[3], f'{what}: counters differ {a[3]} vs {b[3]}'


STEP_CASES = ['neel_oop16', 'neel_oop12x9_pbc', 'neel_oop16_Tfield', 'neel_pin16_perp', 'neel_kagome_perp',
              'neel_oop16_exchange', 'metro_pin32_grid', 'metro_pin24_pbc', 'metro_oop32_trunc_pbc',
              'metro_oop30_trunc', 'metro_oop16_time', 'metro_kagome_grid', 'metro_oop16_single', 'wolff_oop32_pbc',
              'neel_pin16_dimono', 'neel_kagome_dimono', 'metro_sq16_dimono_pbc']


@pytest.mark.parametrize('name', STEP_CASES)
@pytest.mark.parametrize('cs', [1, 2, 4, 8, 16])
def test_engine_equals_step_kernels(name, cs):
    import hotspice_b200 as hs
    if SPECS[name].get('params', {}).get('UPDATE_SCHEME') == 'Wolff' and cs > 2:
        pytest.skip('Wolff runs on the first CTA of a cluster; larger clusters add nothing')
    kw = SPECS[name].get('update_kw', {})
    steps = min(SPECS[name]['steps'], 60)
    a = build_product(name, engine=hs.EngineConfig(persistent=False, use_graphs=False))
    b = build_product(name, engine=hs.EngineConfig(persistent=True, cluster_size=cs))
    a.run(steps, **kw)
    b.run(steps, **kw)
    _assert_same(_state(a), _state(b), f'{name} cs={cs}')


@pytest.mark.parametrize('name', ['progress_oop12', 'progress_pin16_metro'])
@pytest.mark.parametrize('cs', [1, 4, 16])
def test_engine_progress_stop_rule(name, cs):
    import hotspice_b200 as hs
    spec = SPECS[name]
    a = build_product(name, engine=hs.EngineConfig(persistent=False, use_graphs=False))
    b = build_product(name, engine=hs.EngineConfig(persistent=True, cluster_size=cs))
    ra = a.progress(**spec['progress'])
    rb = b.progress(**spec['progress'])
    assert ra == rb
    _assert_same(_state(a), _state(b), f'{name} cs={cs}')


def test_batch_alone_equals_mixed():
    """Each instance gives the same result alone and inside a heterogeneous batch
    (different lattices, sizes, schemes and cluster sizes in one engine call)."""
    import hotspice_b200 as hs
    from hotspice_b200.engine import BatchEngine
    names = ['metro_pin32_grid', 'neel_oop16', 'metro_kagome_grid', 'neel_pin16_perp', 'wolff_oop20_open',
             'metro_oop30_trunc', 'neel_oop12x9_pbc']
    steps = [50, 80, 40, 70, 20, 30, 60]
    cfg = hs.EngineConfig(persistent=True)
    alone = []
    for n, s in zip(names, steps):
        mm = build_product(n, engine=cfg)
        BatchEngine([mm]).run(s, **SPECS[n].get('update_kw', {}))
        alone.append(_state(mm))
    mixed = [build_product(n, engine=cfg) for n in names]
    eng = BatchEngine(mixed)
    # one run() call with per-instance budgets; all instances share the update kwargs of
    # their own scenario, so launch per distinct kwargs
    groups = {}
    for i, n in enumerate(names):
        groups.setdefault(tuple(sorted(SPECS[n].get('update_kw', {}).items())), []).append(i)
    for kw, idx in groups.items():
        sub = BatchEngine([mixed[i] for i in idx])
        sub.run([steps[i] for i in idx], **dict(kw))
    for i, n in enumerate(names):
        _assert_same(alone[i], _state(mixed[i]), f'{n} alone vs mixed')


@pytest.mark.parametrize('cs', [2, 4])
def test_split_clusters_equal_alone(cs, monkeypatch):
    """A launch whose clusters split (HS_INST_ONE_CTA): the unflagged instances run on whole
    clusters, the flagged ones on single CTAs, and every instance ends as it does alone."""
    from hotspice_b200.engine import BatchEngine
    names = ['neel_oop16', 'neel_pin16_perp', 'neel_kagome_perp', 'metro_oop16_single', 'wolff_oop32_pbc',
             'neel_oop12x9_pbc', 'neel_oop16_exchange', 'neel_pin16_dimono']
    steps = [90, 70, 60, 50, 20, 80, 40, 60]
    flags = [False, True, False, True, True, False, True, True]
    alone = []
    for n, s in zip(names, steps):
        mm = build_product(n)
        BatchEngine([mm]).run(s)
        alone.append(_state(mm))
    mixed = [build_product(n) for n in names]
    eng = BatchEngine(mixed, throughput=True)
    monkeypatch.setattr(BatchEngine, '_throughput_sizes', lambda self, st: ([cs] * len(names), flags))
    prepared = eng.run(steps)
    assert len(prepared) == 1 and prepared[0].cs == cs
    # flagged instances come last on the work counter
    assert [flags[j] for j in prepared[0].order] == sorted(flags)
    for i, n in enumerate(names):
        _assert_same(alone[i], _state(mixed[i]), f'{n} cs={cs} one_cta={flags[i]}')


def test_tune_split_leaves_state_and_results():
    """tune_split runs timed launches of candidate plans, restores every instance's state, and
    the tuned plan then gives the same results as an untuned run."""
    from hotspice_b200.engine import BatchEngine
    names = ['neel_oop16', 'neel_pin16_perp', 'metro_oop16_single', 'wolff_oop32_pbc', 'neel_oop12x9_pbc',
             'neel_kagome_perp']
    a = [build_product(n) for n in names]
    b = [build_product(n) for n in names]
    ea, eb = BatchEngine(a, throughput=True), BatchEngine(b, throughput=True)
    ea.run(20)
    eb.run(20)
    before = [_state(x) for x in a]
    cs, k, ms = ea.tune_split(30, reps=1, ks=[1, 3])
    assert cs in (2, 4) and k in (0, 1, 3) and ms > 0
    for n, x, s0 in zip(names, a, before):
        _assert_same(s0, _state(x), f'{n} restored after tuning')
    ea.run(30)
    eb.run(30)
    for n, x, y in zip(names, a, b):
        _assert_same(_state(y), _state(x), f'{n} tuned vs untuned')


def test_captured_graph_replays_equal_direct_launches():
    """A CUDA graph holding one engine launch (BatchEngine.capture) advances a mixed batch
    exactly like direct launches of the same steps."""
    from hotspice_b200.engine import BatchEngine
    names = ['neel_oop16', 'neel_pin16_perp', 'metro_pin32_grid', 'metro_oop30_trunc', 'wolff_oop32_pbc']
    a = [build_product(n) for n in names]
    b = [build_product(n) for n in names]
    ea, eb = BatchEngine(a), BatchEngine(b)
    run = eb.capture(25)
    for _ in range(3):
        ea.run(25)
        run.replay()
    for n, x, y in zip(names, a, b):
        _assert_same(_state(x), _state(y), f'{n} graph replay')


def test_run_from_host_equals_per_array_loads():
    """BatchEngine.run_from_host (one packed copy + scatter kernel in, gather + one copy out) gives
    the same run as loading every array separately and calling run()."""
    import torch
    import hotspice_b200 as hs
    from hotspice_b200.engine import BatchEngine
    names = ['metro_pin32_grid', 'neel_oop16', 'metro_kagome_grid', 'wolff_oop20_open']
    cfg = hs.EngineConfig(persistent=True)
    a = [build_product(n, engine=cfg) for n in names]
    b = [build_product(n, engine=cfg) for n in names]
    ea, eb = BatchEngine(a), BatchEngine(b)
    ea.run(20)
    torch.cuda.synchronize()
    host_in = ea.pack_host()                       # state after 20 steps, packed
    lay, total = ea.state_layout()
    assert host_in.numel() == total
    # b loads the same state array by array
    raw = host_in.numpy()
    for i, f, off, nb in lay:
        t = BatchEngine._field_tensor(b[i], f)
        t.view(-1).view(torch.uint8).copy_(torch.from_numpy(raw[off:off + nb].copy()))
        b[i]._ctl = None
    out_lay, out_total = ea.state_layout(('m', 'C'))
    host_out = torch.empty(out_total, dtype=torch.uint8).pin_memory()
    # the same start state twice: identical results; the second time through the overlapped
    # upload slots
    ea.run_from_host(30, host_in, host_out=host_out)
    torch.cuda.synchronize()
    ea.upload(host_in, slot=1)
    ea.run_from_host(30, slot=1, host_out=host_out)
    torch.cuda.synchronize()
    eb.run(30)
    torch.cuda.synchronize()
    for x, y in zip(a, b):
        _assert_same(_state(x), _state(y), 'run_from_host')
    from hotspice_b200 import _lib
    ho = host_out.numpy()
    for i, f, off, nb in out_lay:
        ref = BatchEngine._field_tensor(b[i], f).view(-1).view(torch.uint8).cpu().numpy()
        if f == 'C':   # every counter but the Wolff stamp epoch (it counts clusters ever grown)
            x = np.frombuffer(ho[off:off + nb].tobytes(), dtype=_lib.COUNTERS_DTYPE)[0]
            y = np.frombuffer(ref.tobytes(), dtype=_lib.COUNTERS_DTYPE)[0]
            assert all(np.array_equal(x[k], y[k]) for k in _lib.COUNTERS_DTYPE.names if k != 'epoch'), i
        else:
            assert np.array_equal(ho[off:off + nb], ref), (i, f)


@pytest.mark.parametrize('name', ['progress_oop12', 'progress_pin16_metro'])
def test_progress_launch_budget(name):
    """A progress() launch ends after its step budget with done = 0 (every launch ends, however
    far the stop rule is); BatchEngine.progress continues the run over further launches, and
    the result equals a run made in one launch, bit for bit."""
    import hotspice_b200 as hs
    from hotspice_b200.engine import BatchEngine
    spec = SPECS[name]
    # one launch with a 5-step budget and a stop rule far away: exactly 5 steps, not done
    c = build_product(name, engine=hs.EngineConfig(persistent=True, cluster_size=1))
    c._write_counters(t0=0.0, mc0=0.0, t_max=1e30, mc_max=1e12, progress=1, done=0)
    s0 = int(c._read_counters()['steps'])
    eng = BatchEngine([c], cluster_size=1)
    eng.launch(eng._prepare([5], [{}]))
    r = c._read_counters()
    assert int(r['steps']) - s0 == 5 and int(r['done']) == 0 and int(r['status']) == 0
    c._write_counters(progress=0, done=0)
    # the same progress() split into launches of 3 steps, and in one launch
    a = build_product(name, engine=hs.EngineConfig(persistent=True, cluster_size=1))
    b = build_product(name, engine=hs.EngineConfig(persistent=True, cluster_size=1))
    ea, eb = BatchEngine([a], cluster_size=1), BatchEngine([b], cluster_size=1)
    ea.progress_launch_steps = 3
    ra = ea.progress(**spec['progress'])
    rb = eb.progress(**spec['progress'])
    assert ea.launches > 1 and eb.launches == 1
    assert ra == rb
    _assert_same(_state(a), _state(b), f'{name} budget 3 vs one launch')


def test_armed_progress_that_hits_its_budget_is_reported():
    """A device-armed progress() (hs_progress_arm + engine launch, as the reservoir I/O uses)
    whose launch ends at its step budget is flagged HS_ST_STEP_CAP by the next disarm, so the
    host raises instead of reading a truncated run."""
    import hotspice_b200 as hs
    from hotspice_b200 import _lib
    from hotspice_b200.engine import BatchEngine
    a = build_product('progress_oop12', engine=hs.EngineConfig(persistent=True, cluster_size=1))
    a._progress_arm(t_max=1e30, MCsteps_max=1e12)
    eng = BatchEngine([a], cluster_size=1)
    eng.launch(eng._prepare([4], [{}]))
    with pytest.raises(RuntimeError, match='status 16'):
        a._progress_finish()
    assert int(a._read_counters()['status']) & _lib.HS_ST_STEP_CAP
    a._write_counters(status=0)


def _bench_like(k, n=48, scheme='Metropolis'):
    import hotspice_b200 as hs
    lat = (hs.ASI.OOP_Square, hs.ASI.IP_Pinwheel)[k % 2]
    a = (200e-9, 300e-9)[k % 2]
    g = np.random.Generator(np.random.PCG64(40 + k))
    return lat(a, n, T=300.0, E_B=5.5e-20 * g.lognormal(0, 0.05, size=(n, n)), moment=1.1e-15 if k % 2 == 0 else 1e-15,
               pattern=g.integers(0, 2, size=(n, n)) * 2 - 1, seed=40 + k,
               energies=[hs.DipolarEnergy(cutoff_range=16 * a), hs.ZeemanEnergy(2e-3, 0.3)],
               params=hs.SimParams(UPDATE_SCHEME=scheme))


def test_batch_resync_bounds_drift():
    """BatchEngine.run(..., resync_every=R) recomputes every instance's energies after each R
    steps: right after a resync the incremental energies equal a fresh FP64 recompute, and
    R steps later they are within 1e-6 of one (the FP32 increments' drift)."""
    from hotspice_b200.engine import BatchEngine
    mms = [_bench_like(k, scheme=('Neel', 'Metropolis')[k % 2]) for k in range(4)]
    eng = BatchEngine(mms)
    eng.run(200, resync_every=100)               # ends on a resync
    for mm in mms:
        assert mm.resync_energies(measure=True) == 0.0
    eng.run(250, resync_every=100)               # 50 steps since the last resync
    for mm in mms:
        if mm._dipolar().kernel_set.asymmetry < 1e-12:
            assert mm.resync_energies(measure=True) <= 1e-6


def test_captured_resync_equals_direct_run():
    """The CUDA graph of a run with resyncs (engine launches and recomputes) replays the same
    states as BatchEngine.run with the same resync_every."""
    from hotspice_b200.engine import BatchEngine
    a = [_bench_like(k) for k in range(3)]
    b = [_bench_like(k) for k in range(3)]
    BatchEngine(a).run(150, resync_every=60)
    g = BatchEngine(b).capture(150, resync_every=60)
    g.replay()
    for x, y in zip(a, b):
        _assert_same(_state(x), _state(y), 'captured resync')


def test_server_resync():
    """Server(resync_every=R) recomputes a request's energies after each R of its own steps
    (quanta are cut there), so the results are the same alone and in the mix, bit for bit."""
    import torch
    from hotspice_b200 import serving as SV
    reqs = [SV.SimRequest(i, dict(lattice=('OOP_Square', 'IP_Pinwheel')[i % 2], n=40 + 8 * i, T=300.0, B=1e-3,
                                  angle=0.2, scheme=('Neel', 'Metropolis')[i % 2], seed=900 + i), 250 + 40 * i, 0.0)
            for i in range(4)]
    dev = torch.device('cuda')
    mix = {r.rid: r for r in SV.Server(device=dev, keep_state=True, resync_every=64, round_ms=0.3).serve(reqs, realtime=False)}
    for q in reqs:
        alone = SV.Server(device=dev, keep_state=True, resync_every=64, round_ms=2.0).serve([q], realtime=False)[0]
        got = mix[q.rid]
        assert np.array_equal(alone.state, got.state), q.rid
        assert (alone.switches, alone.attempts, alone.t) == (got.switches, got.attempts, got.t)
        assert alone.E_tot == got.E_tot


@pytest.mark.parametrize('r_cells', [4, 1])
def test_poisson_workspace_does_not_change_results(r_cells, monkeypatch):
    """A Poisson-disc instance gives the same state whether the engine launch keeps its
    sampler arrays in shared memory (workspace sized by poisson_workspace) or in the
    instance's scratch (workspace 0), and the same as the per-step kernels. At r = 1a the
    96 x 96 background grid (68 x 68 cells, 111 KB) still fits; at r = 4a it is 28 x 28."""
    import hotspice_b200 as hs
    import hotspice_b200.engine as E
    a, n = 200e-9, 96
    g = np.random.Generator(np.random.PCG64(31))
    spec = {'lattice': 'OOP_Square', 'a': a, 'moment': 1e-15, 'nx': n, 'ny': n, 'seed': 31, 'kw': {'PBC': True},
            'energies': [{'type': 'dipolar', 'cutoff': 6 * a}, {'type': 'zeeman', 'B': 1e-3, 'angle': 0.0}],
            'params': {'UPDATE_SCHEME': 'Metropolis', 'MULTISAMPLING_SCHEME': 'Poisson'}}
    fx = {'T': 300.0, 'E_B': 5e-20 * np.ones((n, n)), 'm0': g.integers(0, 2, size=(n, n)) * 2 - 1}
    kw = {'r': r_cells * a}
    steps = 30
    ref = build_product('ws_ref', spec=spec, fx=fx, engine=hs.EngineConfig(persistent=False, use_graphs=False))
    ref.run(steps, **kw)
    shared = build_product('ws_shared', spec=spec, fx=fx, engine=hs.EngineConfig(persistent=True))
    prep = E.BatchEngine([shared]).run(steps, **kw)
    assert prep[0].ws > 0, 'the sampler arrays should fit the workspace'
    monkeypatch.setattr(E, 'poisson_workspace', lambda I: 0)
    scratch = build_product('ws_scratch', spec=spec, fx=fx, engine=hs.EngineConfig(persistent=True))
    prep2 = E.BatchEngine([scratch]).run(steps, **kw)
    assert prep2[0].ws == 0
    sr = _state(ref)
    _assert_same(sr, _state(shared), f'r={r_cells}a shared workspace')
    _assert_same(sr, _state(scratch), f'r={r_cells}a scratch')


def test_engine_reports_device_time_per_instance():
    """hs_engine_run_ws writes each instance's device time: a permutation of the instances
    over the launch slots, every time positive, and longer runs take longer."""
    from hotspice_b200.engine import BatchEngine
    names = ['neel_oop16', 'metro_pin32_grid', 'neel_pin16_perp', 'metro_oop30_trunc']
    mms = [build_product(n) for n in names]
    eng = BatchEngine(mms, cluster_size=1)
    prep = eng.run([40, 40, 40, 400])
    ns = {}
    for p in prep:
        assert sorted(p.order) == list(range(p.n)) or len(prep) > 1
        for slot, j in enumerate(p.order):
            ns[j] = int(p.ns[slot].item())
    assert sorted(ns) == list(range(len(names)))
    assert all(v > 0 for v in ns.values()), ns
    prep = eng.run([40, 40, 40, 4000])
    long = {j: int(p.ns[s].item()) for p in prep for s, j in enumerate(p.order)}
    assert long[3] > ns[3], (long[3], ns[3])
