"""Host-side serving policy (no GPU): admission by HBM footprint and slots, round quanta,
FIFO latency model, the seeded request stream, and the per-rank sharding of the stream,
including a two-rank gloo run that checks the ranks agree on a disjoint, complete split."""
import os
import time
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from hotspice_b200 import serving as S


def _req(rid, n, steps=1000, lattice='OOP_Square', arrival=0.0):
    return S.SimRequest(rid, dict(lattice=lattice, n=n, T=300.0, seed=rid), steps, arrival)


def test_request_stream_is_seeded_and_poisson():
    a = S.request_stream(2000, rate=200.0, seed=3)
    b = S.request_stream(2000, rate=200.0, seed=3)
    assert [(r.spec, r.steps, r.arrival) for r in a] == [(r.spec, r.steps, r.arrival) for r in b]
    gaps = np.diff([0.0] + [r.arrival for r in a])
    assert abs(gaps.mean() - 1 / 200.0) < 0.1 / 200.0          # mean inter-arrival 5 ms
    ns = np.array([r.spec['n'] for r in a])
    steps = np.array([r.steps for r in a])
    assert ns.min() >= 64 and ns.max() <= 1024
    assert steps.min() >= 1000 and steps.max() <= 100000
    # log-uniform: the median sits near the geometric mean of the range
    assert abs(np.log(np.median(steps)) - np.log(1e4)) < 0.25
    assert {r.spec['lattice'] for r in a} == {'OOP_Square', 'IP_Pinwheel', 'IP_Kagome', 'Ising_Square'}


def test_footprint_grows_with_cells():
    small = S.footprint_bytes(dict(lattice='OOP_Square', n=64))
    big = S.footprint_bytes(dict(lattice='OOP_Square', n=1024))
    assert big > small * 20
    assert S.footprint_bytes(dict(lattice='IP_Pinwheel', n=256)) > S.footprint_bytes(dict(lattice='OOP_Square', n=256))


def test_admission_respects_bytes_and_slots():
    q = S.AdmissionQueue(footprint=lambda spec: spec['n'])
    for i, n in enumerate([5, 3, 4, 1]):
        q.push(_req(i, n))
    got = q.admit(free_bytes=8, free_slots=10)
    assert [r.rid for r in got] == [0, 1]          # 5 + 3 fill the 8 bytes
    assert [r.rid for r in q.waiting] == [2, 3]
    assert [r.rid for r in q.admit(free_bytes=2, free_slots=10)] == [3]   # 1 passes the 4 that does not fit
    q2 = S.AdmissionQueue(footprint=lambda spec: 1)
    for i in range(5):
        q2.push(_req(i, 1))
    assert len(q2.admit(free_bytes=100, free_slots=2)) == 2
    assert len(q2) == 3


def test_admission_bypass_is_bounded():
    q = S.AdmissionQueue(footprint=lambda spec: spec['n'], max_skip=2)
    q.push(_req(0, 10))                            # too big for now
    for i in range(1, 6):
        q.push(_req(i, 1))
    assert [r.rid for r in q.admit(3, 100)] == [1, 2, 3]   # small ones pass the big head
    assert [r.rid for r in q.admit(1, 100)] == [4]
    assert q.admit(1, 100) == []                   # passed over 3 times: the head now blocks
    assert [r.rid for r in q.admit(11, 100)] == [0, 5]


def test_plan_quanta():
    steps = S.plan_quanta([10.0, 100.0, 1e4], [50, 1000, 7], round_us=1000.0)
    assert steps == [50, 10, 1]                    # capped by what remains; at least one step


def test_plan_quanta_lengthens_the_critical_runs():
    # 300 short runs and one long one on 148 SMs: the long run's remaining 2 s exceed the drain
    # time of the resident work, so its quantum grows in proportion, up to the round's length
    times = [10.0] * 300 + [100.0]
    remaining = [400] * 300 + [20000]
    sizes = [1] * 300 + [16]
    steps = S.plan_quanta(times, remaining, 1000.0, sizes, 148)
    assert steps[:300] == [100] * 300              # round_us / 10 us
    rem_us = [r * t for r, t in zip(remaining, times)]
    drain = sum(x * c for x, c in zip(rem_us, sizes)) / 148
    W = max(1000.0, sum(min(1000.0, x) * c for x, c in zip(rem_us, sizes)) / 148)
    assert steps[300] == int(min(W, W * rem_us[300] / drain) // 100.0)
    assert 10 < steps[300] <= W / 100.0 + 1
    # without the sizes, every run gets the plain quantum
    assert S.plan_quanta(times, remaining, 1000.0)[300] == 10


def test_plan_sizes():
    from hotspice_b200.engine import plan_sizes, plan_uniform_size, lpt_makespan
    neel_big = (9.0, 600.0, 0.62)                   # ~500^2-cell Néel lattice
    neel_small = (9.0, 2.0, 0.62)
    wolff = (12.0, 0.0, 0.0)                        # grows on one CTA: never widened
    # one long run among short ones gets a wide cluster; short runs stay on one CTA
    cs = plan_sizes([neel_big] + [neel_small] * 200, [5000] + [100] * 200, n_sm=148)
    assert cs[0] >= 8 and set(cs[1:]) == {1}
    assert plan_sizes([wolff] * 3, [10**6] * 3, n_sm=148) == [1, 1, 1]
    # many equal runs that fill the GPU: one CTA each
    assert plan_sizes([neel_big] * 300, [100] * 300, n_sm=148) == [1] * 300
    # widening stops when it no longer shortens the run by 20%
    assert plan_sizes([(9.0, 2.0, 0.62)], [10**6], n_sm=148) == [1]
    # one size per launch: a few long runs want wide clusters, many short ones want one CTA each
    assert plan_uniform_size([neel_big] * 4, [10**4] * 4, n_sm=148) >= 8
    assert plan_uniform_size([neel_small] * 600, [100] * 600, n_sm=148) == 1
    assert lpt_makespan([5, 4, 3, 3, 3], 2) == 10


def test_plan_split():
    """One launch whose long runs use whole clusters and whose short runs take one CTA each."""
    from hotspice_b200.engine import lpt_makespan, model_time, plan_split, split_makespan
    workers = {1: 148, 2: 74, 4: 37, 8: 18, 16: 9}
    neel_big = (9.0, 600.0, 0.62)
    neel_small = (9.0, 2.0, 0.62)
    # two clusters of 2: cluster runs 10 and 6 on separate clusters, then the CTAs (free at
    # 6, 6, 10, 10) take 5 and 4 (ending at 11 and 10), and the 3s end at 13
    assert split_makespan([10, 6], [5, 4, 3, 3], 2, 2) == 13
    # a few long runs among many short ones: the long ones use clusters, the rest one CTA
    models = [neel_big] * 6 + [neel_small] * 400
    steps = [2000] * 6 + [200] * 400
    cs, flags, mk = plan_split(models, steps, workers)
    assert cs > 1 and not any(flags[:6]) and all(flags[6:])
    uniform = min(max(st * model_time(m, c) for m, st in zip(models, steps)) for c in (2, 4, 8, 16))
    assert mk <= uniform
    # equal short runs that fill the GPU: no worse than one CTA each
    cs, flags, mk = plan_split([neel_small] * 600, [100] * 600, workers)
    assert mk <= lpt_makespan([100 * model_time(neel_small, 1)] * 600, 148)
    assert cs == 1 or sum(flags) >= 500
    # a single long run: one wide cluster, nothing on one CTA
    cs, flags, _ = plan_split([neel_big], [10**4], workers)
    assert cs >= 8 and flags == [False]


def test_fifo_latencies():
    lat = S.fifo_latencies([0.0, 0.1, 0.2], [0.5, 0.1, 0.1])
    assert np.allclose(lat, [0.5, 0.5, 0.5])


def test_shard_requests_partition():
    reqs = S.request_stream(300, seed=5)
    shards = [S.shard_requests(reqs, 3, r) for r in range(3)]
    ids = sorted(x.rid for s in shards for x in s)
    assert ids == list(range(300))
    loads = [sum(x.steps * (S.geometry_shape(x.spec)[0] * S.geometry_shape(x.spec)[1] + 1089) for x in s) for s in shards]
    assert max(loads) <= 1.5 * min(loads)


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        reqs = S.request_stream(200, seed=11)
        mine = [r.rid for r in S.shard_requests(reqs, world, rank)]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        if rank == 0:
            out.put(gathered)
    finally:
        dist.destroy_process_group()


def test_shard_requests_two_ranks_gloo():
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    a, b = map(set, gathered)
    assert not (a & b)
    assert a | b == set(range(200))
    assert abs(len(a) - len(b)) < 100


def _dealer_stream():
    """120 equal requests, one every millisecond."""
    return [S.SimRequest(i, dict(lattice='OOP_Square', n=64, T=300.0, seed=i), 1000, 1e-3 * i) for i in range(120)]


def _dealer_main(rank, world, port, drain, realtime, out):
    """One rank of a simulated serving run: held work drains at ``drain[rank]`` requests per
    second of the shared clock, and the rank claims arrived requests through a RequestDealer
    on a shared TCPStore."""
    import datetime
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        store = dist.TCPStore('127.0.0.1', port + 1, world, rank == 0, timeout=datetime.timedelta(seconds=60))
        reqs = _dealer_stream()
        unit = S.request_work(reqs[0])
        dealer = S.RequestDealer(reqs, store, rank, world, grace_s=0.02, poll_s=0.0)
        dist.barrier()
        t0 = last = time.perf_counter()
        held, got = 0.0, []
        while not dealer.exhausted() or held > 0:
            t = time.perf_counter()
            held = max(0.0, held - drain[rank] * unit * (t - last))
            last = t
            for r in dealer.claim(t - t0 if realtime else float('inf'), held):
                got.append(r.rid)
                held += S.request_work(r)
            time.sleep(2e-4)
        gathered = [None] * world
        dist.all_gather_object(gathered, got)
        if rank == 0:
            out.put(gathered)
    finally:
        dist.destroy_process_group()


def test_request_dealer_one_rank_follows_arrivals():
    """One rank on a local store: arrived requests are dealt in arrival order and nothing that
    has not arrived yet; the shared index records the claimer."""
    import datetime
    store = dist.TCPStore('127.0.0.1', _free_port(), 1, True, timeout=datetime.timedelta(seconds=30))
    reqs = _dealer_stream()[:10]
    d = S.RequestDealer(list(reversed(reqs)), store, 0, 1, poll_s=0.0)
    assert [r.rid for r in d.claim(0.0035, 0.0)] == [0, 1, 2, 3]
    assert d.claim(0.0035, 0.0) == [] and not d.exhausted()
    assert [r.rid for r in d.claim(1.0, 0.0)] == list(range(4, 10))
    assert d.exhausted() and store.get('hs_dealer/next').decode() == '10:0'
    assert d.claim(2.0, 0.0) == []


@pytest.mark.parametrize('realtime', [True, False])
def test_request_dealer_two_ranks_gloo(realtime):
    """Run-time placement over two gloo ranks: every request is dealt exactly once, each rank
    receives its requests in arrival order, and the rank that works its load off ten times
    faster receives more of them."""
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_dealer_main, args=(r, 2, port, [500.0, 50.0], realtime, q)) for r in range(2)]
    for p in procs:
        p.start()
    gathered = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    a, b = gathered
    assert sorted(a + b) == list(range(120))
    assert a == sorted(a) and b == sorted(b)
    assert len(a) > len(b)


def test_segment_table_covers_packed_layout():
    """The HsSegment table of the packed batch transfer: every array covered exactly once, pieces
    of at most HS_SEGMENT_MAX bytes, staged and device sides advancing together, 16-byte
    aligned piece starts when both bases are aligned (the kernel's vector path), and the
    struct layout of the C header (24 bytes)."""
    from hotspice_b200 import _lib
    from hotspice_b200.engine import SEGMENT_DTYPE, segment_table
    assert SEGMENT_DTYPE.itemsize == 24
    import ctypes
    sizes = (ctypes.c_int32 * 7)()
    _lib.load().hs_struct_sizes(sizes, 7)
    assert sizes[6] == SEGMENT_DTYPE.itemsize          # the library's sizeof(HsSegment)
    sizes = [1, 15, 16, 1000, 65536, 65537, 300000]
    layout, off = [], 0
    for i, nb in enumerate(sizes):
        layout.append((i, 'x', off, nb))
        off += -(-nb // 256) * 256
    ptrs = [0x7f0000000000 + 0x100000 * i for i in range(len(sizes))]
    rows = segment_table(layout, ptrs)
    assert np.all(rows['bytes'] > 0) and np.all(rows['bytes'] <= _lib.HS_SEGMENT_MAX)
    for (i, _, o, nb), p in zip(layout, ptrs):
        mine = rows[(rows['device'] >= p) & (rows['device'] < p + nb)]
        assert int(mine['bytes'].sum()) == nb
        assert np.all(mine['staged'] - o == mine['device'] - p)
        assert np.all(mine['staged'] % 16 == 0) and np.all(mine['device'] % 16 == 0)
    small = segment_table(layout, ptrs, max_bytes=4096)
    assert int(small['bytes'].sum()) == sum(sizes) and np.all(small['bytes'] <= 4096)
