"""Continuous-batching server on the GPU: every request gives the same result alone, in a
mix that arrives while others are on the device, and through the plain per-step kernels;
the HBM budget bounds how many requests are resident at once."""
import numpy as np
import pytest

from hotspice_b200 import serving as S

pytestmark = pytest.mark.gpu


def _requests():
    specs = [
        dict(lattice='OOP_Square', n=40, T=300.0, B=1e-3, angle=0.3, scheme='Neel', seed=101),
        dict(lattice='IP_Pinwheel', n=32, T=250.0, B=2e-3, angle=1.1, scheme='Metropolis', seed=102),
        dict(lattice='IP_Kagome', n=36, T=350.0, B=0.0, angle=0.0, scheme='Neel', seed=103),
        dict(lattice='Ising_Square', n=24, T=180.0, seed=104, J=1e-21),
        dict(lattice='OOP_Square', n=64, T=220.0, B=4e-3, angle=2.0, scheme='Metropolis', seed=105),
        dict(lattice='IP_Pinwheel', n=48, T=390.0, B=5e-3, angle=4.0, scheme='Neel', seed=106),
    ]
    steps = [600, 300, 900, 40, 250, 1200]
    return [S.SimRequest(i, s, st, arrival=0.002 * i) for i, (s, st) in enumerate(zip(specs, steps))]


def _check_same(a, b):
    assert a.rid == b.rid
    assert np.array_equal(a.state, b.state)
    assert a.switches == b.switches and a.attempts == b.attempts
    assert abs(a.E_tot - b.E_tot) <= 1e-6 * max(abs(b.E_tot), 1e-30)
    assert a.t == pytest.approx(b.t, rel=1e-12, abs=0)


def test_alone_equals_mix_equals_plain():
    import torch
    reqs = _requests()
    alone = {}
    for r in reqs:
        res = S.Server(keep_state=True).serve([r], realtime=False)
        assert len(res) == 1
        alone[r.rid] = res[0]
    # the mix: staggered arrivals, short rounds, so later requests join while others run
    srv = S.Server(keep_state=True, round_ms=0.05)
    mix = {r.rid: r for r in srv.serve(reqs, realtime=True)}
    assert sorted(mix) == [r.rid for r in reqs]
    assert srv.stats.rounds > 1 and srv.stats.max_active > 1
    for r in reqs:
        _check_same(mix[r.rid], alone[r.rid])
    # the plain form: per-step kernels replayed from CUDA graphs, one instance at a time
    for r in reqs:
        mm = S.build_magnets(r.spec)
        mm.engine.persistent = False
        mm.run(r.steps)
        torch.cuda.synchronize()
        assert np.array_equal(mm._m_dev.cpu().numpy(), alone[r.rid].state)
        assert abs(mm.E_tot - alone[r.rid].E_tot) <= 1e-6 * max(abs(mm.E_tot), 1e-30)


def test_hbm_budget_limits_residency():
    reqs = _requests()
    budget = sum(sorted(S.footprint_bytes(r.spec) for r in reqs)[-2:])
    srv = S.Server(keep_state=True, hbm_budget=budget, round_ms=0.05)
    res = srv.serve(reqs, realtime=False)
    assert len(res) == len(reqs)
    assert srv.stats.admitted_bytes_peak <= budget
    assert srv.stats.max_active <= 2
    ref = {r.rid: S.Server(keep_state=True).serve([r], realtime=False)[0] for r in reqs[:2]}
    got = {r.rid: r for r in res}
    for rid, a in ref.items():
        _check_same(got[rid], a)


def test_request_too_large_for_budget_raises():
    r = _requests()[0]
    with pytest.raises(RuntimeError, match='HBM budget'):
        S.Server(hbm_budget=1024).serve([r], realtime=False)


def test_building_a_request_does_not_synchronise():
    """A request's Magnets is built without the host waiting on the device (pinned
    asynchronous uploads, no read-backs), so the server's builder threads never stall behind
    the engine rounds that hold the SMs."""
    import torch
    specs = [dict(lattice='OOP_Square', n=70, T=300.0, B=1e-3, angle=0.3, scheme='Neel', seed=201),
             dict(lattice='IP_Pinwheel', n=64, T=250.0, B=2e-3, angle=1.1, scheme='Metropolis', seed=202),
             dict(lattice='IP_Kagome', n=66, T=350.0, B=0.0, angle=0.0, scheme='Neel', seed=203),
             dict(lattice='Ising_Square', n=48, T=180.0, seed=204, J=1e-21)]
    for s in specs:
        S.build_magnets(s)          # first build of each kind: library load, lazy set-up
    torch.cuda.synchronize()
    torch.cuda.set_sync_debug_mode('error')
    try:
        built = [S.build_magnets(dict(s, seed=s['seed'] + 10)) for s in specs]
    finally:
        torch.cuda.set_sync_debug_mode('default')
    torch.cuda.synchronize()
    for mm in built:   # and the instances are complete: a summary reads back normally
        assert np.isfinite(mm.E_tot)


def test_served_through_a_dealer_equals_alone():
    """Server.serve with a RequestDealer (one rank on a local store) serves every request of
    the stream, each with the same result as alone."""
    import datetime
    import socket
    import torch.distributed as dist
    reqs = _requests()
    alone = {r.rid: S.Server(keep_state=True).serve([r], realtime=False)[0] for r in reqs}
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        port = s.getsockname()[1]
    store = dist.TCPStore('127.0.0.1', port, 1, True, timeout=datetime.timedelta(seconds=60))
    dealer = S.RequestDealer(reqs, store, 0, 1)
    srv = S.Server(keep_state=True, round_ms=0.05)
    got = {r.rid: r for r in srv.serve([], realtime=True, dealer=dealer)}
    assert sorted(got) == [r.rid for r in reqs]
    for r in reqs:
        _check_same(got[r.rid], alone[r.rid])
