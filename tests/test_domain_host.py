"""Domain decomposition of one lattice (hotspice_b200/domain.py) on CPU: the slab and halo
bookkeeping as pure functions, and two gloo ranks whose stitched results equal one process's:
a windowed energy recompute of the owned rows after a halo exchange, the window update of a
step's switches gathered in list order, and the global Néel argmin. The arithmetic here is a
plain restatement of the windowed sums (the same loops on both sides, so equal bit for bit);
on GPUs the slabs hold device arrays and the same collectives run over NCCL (not measured on
hardware: every run here has one GPU)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from hotspice_b200 import domain as D


def test_partition_rows_covers_and_aligns():
    for ny, world, halo, pbc, unit in ((24, 2, 3, True, 1), (24, 3, 4, False, 2), (40, 4, 5, True, 4), (7, 1, 3, True, 1)):
        sl = D.partition_rows(ny, 10, world, halo, pbc, unit)
        own = np.concatenate([np.arange(s.r0, s.r1) for s in sl])
        assert np.array_equal(own, np.arange(ny))
        for s in sl:
            assert s.r0 % unit == 0 and s.r1 % unit == 0 and s.h % unit == 0
            if world > 1:
                assert s.h >= halo
            rows = s.rows
            assert np.array_equal(rows[s.own], np.arange(s.r0, s.r1))
            assert len(rows) == (s.r1 - s.r0) + s.lo + s.hi
            if not pbc and world > 1:
                assert rows.min() >= 0 and rows.max() < ny
            assert (s.r0 - s.lo) % unit == 0          # local row 0 starts a unit cell
    with pytest.raises(ValueError):
        D.partition_rows(10, 4, 4, 3, True)           # slabs thinner than the halo
    with pytest.raises(ValueError):
        D.partition_rows(9, 4, 2, 1, True, unit=2)    # rows not whole unit cells


def test_slab_switches_picks_the_reaching_switches():
    s = D.partition_rows(24, 8, 2, 3, True)[0]      # owns rows 0..11, halo rows 21..23 and 12..14
    sw = np.array([[0, 22, 1], [1, 5, 2], [2, 14, 3], [3, 15, 4], [4, 18, 5]])
    loc = D.slab_switches(sw, s, 3)
    # rows 22 (wraps to -2), 5 and 14 reach rows 0..11 within 3; 15 and 18 do not
    assert loc.tolist() == [[s.local_row(22), 1], [s.local_row(5), 2], [s.local_row(14), 3]]


# ---------------------------------------------------------------------------- two ranks
NY, NX, W = 24, 20, 3


def _problem(pbc):
    g = np.random.Generator(np.random.PCG64(5 + pbc))
    mm = g.choice([-1.0, 1.0], size=(NY, NX)) * 1e-15
    K = g.normal(size=(2 * W + 1, 2 * W + 1)) * 1e10
    K[W, W] = 0.0
    sw = np.array([[k, int(g.integers(0, NY)), int(g.integers(0, NX))] for k in range(12)])
    sw[:, 1][:4] = [0, NY - 1, NY // 2 - 1, NY // 2]       # near the slab edges
    keys = g.random((NY, NX))
    keys[3, 4] = keys[NY - 2, 7] = -1.0                     # a tie across the two slabs
    return mm, K, sw, keys


def _window_sum(src, K, rows, cols_n, pbc, y, x, y_of):
    """sum over the window of K(d) * src at (y + dy, x + dx); src rows are indexed through
    y_of (global row -> row of src, None when absent)."""
    acc = 0.0
    for dy in range(-W, W + 1):
        yy = y + dy
        if pbc:
            yy %= NY
        elif not 0 <= yy < NY:
            continue
        r = y_of(yy)
        for dx in range(-W, W + 1):
            xx = x + dx
            if pbc:
                xx %= NX
            elif not 0 <= xx < NX:
                continue
            acc += K[dy + W, dx + W] * src[r, xx]
    return acc


def _energies(src, K, pbc, rows, y_of):
    return np.array([[_window_sum(src, K, None, NX, pbc, y, x, y_of) for x in range(NX)] for y in rows])


def _update(E, mm, K, sw_list, rows, pbc, y_of):
    """E_j += 2 mm_j sum_s mm_s K(j - s) over the switches in list order (update_multiple)."""
    E = E.copy()
    for j, y in enumerate(rows):
        for x in range(NX):
            acc = 0.0
            for sy, sx in sw_list:
                dy, dx = y - sy, x - sx
                if pbc:
                    dy = (dy + NY // 2) % NY - NY // 2
                    dx = (dx + NX // 2) % NX - NX // 2
                if abs(dy) <= W and abs(dx) <= W:
                    acc += mm[y_of(sy), sx] * K[dy + W, dx + W]
            E[j, x] += 2 * mm[y_of(y), x] * acc
    return E


def _rank_main(rank, world, port, pbc, q):
    os.environ.update(MASTER_ADDR='127.0.0.1', MASTER_PORT=str(port))
    dist.init_process_group('gloo', rank=rank, world_size=world)
    try:
        mm, K, sw, keys = _problem(pbc)
        slab = D.partition_rows(NY, NX, world, W, pbc)[rank]
        local = torch.zeros((len(slab.rows), NX), dtype=torch.float64)
        local[slab.own] = torch.from_numpy(mm[slab.r0:slab.r1])     # only the owned rows are known
        D.exchange_halo(local, slab)
        src = local.numpy()
        own_rows = range(slab.r0, slab.r1)
        E = _energies(src, K, pbc, own_rows, slab.local_row)
        # this rank's switches are those in its rows; all ranks merge them in list order
        mine = torch.from_numpy(sw[(sw[:, 1] >= slab.r0) & (sw[:, 1] < slab.r1)])
        allsw = D.gather_switches(mine)
        loc = D.slab_switches(allsw, slab, W)
        glob = [(int(slab.rows[ly]), x) for ly, x in loc]
        E2 = _update(E, src, K, glob, own_rows, pbc, slab.local_row)
        # Néel: this rank's minimum, then the global one
        kk = keys[slab.r0:slab.r1]
        i = int(np.argmin(kk))
        best = D.global_argmin(float(kk.flat[i]), slab.r0 * NX + i)
        q.put((rank, slab.r0, slab.r1, E, E2, allsw.numpy(), best))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


@pytest.mark.parametrize('pbc', [True, False])
def test_two_ranks_equal_one_process(pbc):
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, pbc, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=180) for _ in range(2)])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    mm, K, sw, keys = _problem(pbc)
    ident = lambda y: y  # noqa: E731
    E_one = _energies(mm, K, pbc, range(NY), ident)
    E2_one = _update(E_one, mm, K, [(int(y), int(x)) for _, y, x in sw], range(NY), pbc, ident)
    E = np.concatenate([r[3] for r in res])
    E2 = np.concatenate([r[4] for r in res])
    assert np.array_equal(E, E_one)
    assert np.array_equal(E2, E2_one)
    for r in res:
        assert np.array_equal(r[5], sw)                         # single-process list order
        flat = int(np.argmin(keys))
        assert r[6] == (float(keys.flat[flat]), flat)           # ties to the smaller index
