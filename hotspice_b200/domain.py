"""Domain decomposition of one lattice over several ranks (one process per GPU).

A lattice too large for one device, or one that should advance faster than one device allows,
is cut into horizontal slabs of whole unit-cell rows, one per rank. A rank keeps its own rows
plus a halo of ``h`` rows on each side, ``h`` the half-height of the dipolar window, so every
source whose window reaches an owned row is present locally:

* a full or windowed energy recompute of the owned rows needs the halo rows of m * moment,
  refreshed by :func:`exchange_halo` (each rank sends its first and last ``h`` owned rows to
  its neighbours; periodic lattices wrap around);
* an update step's switches are gathered from every rank (:func:`gather_switches`) in the
  order a single process would list them (the order fixes the FP32 summation order of the
  window update, hotspice/energies.py:331-366), and each rank applies those whose window
  reaches its rows (:func:`slab_switches` gives them in the slab's own coordinates, the input
  of hs_dipolar_update on the slab's arrays);
* a Néel step (hotspice/core.py:679-709) picks the global minimum of the per-rank minima of
  the log-domain keys (:func:`global_argmin`), ties to the smaller row-major index like
  numpy's nanargmin.

The collectives go through torch.distributed, so the same code runs on gloo (host tensors)
and on NCCL (device tensors). Slabs are aligned to the unit cell so that a slab's sublattice
pattern is the lattice's own.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class Slab:
    """The rows one rank holds: owned rows [r0, r1) and ``h`` halo rows on each side; local row
    j is global row ``rows[j]`` (periodic wrap when ``pbc``; clipped at open edges)."""
    rank: int
    world: int
    ny: int
    nx: int
    r0: int
    r1: int
    h: int
    pbc: bool

    @property
    def lo(self) -> int:
        """Halo rows below r0 that exist (all h with PBC or away from the edge)."""
        return self.h if (self.pbc or self.world == 1) else min(self.h, self.r0)

    @property
    def hi(self) -> int:
        return self.h if (self.pbc or self.world == 1) else min(self.h, self.ny - self.r1)

    @property
    def rows(self) -> np.ndarray:
        """Global row of each local row."""
        g = np.arange(self.r0 - self.lo, self.r1 + self.hi)
        return g % self.ny if self.pbc else g

    @property
    def own(self) -> slice:
        """Local rows that this rank owns."""
        return slice(self.lo, self.lo + (self.r1 - self.r0))

    def local_row(self, y: int) -> int | None:
        """Local index of global row y (None when this slab does not hold it)."""
        d = y - (self.r0 - self.lo)
        if self.pbc:
            d %= self.ny
        n = self.r1 - self.r0 + self.lo + self.hi
        return d if 0 <= d < n else None


def partition_rows(ny: int, nx: int, world: int, halo: int, pbc: bool, unit: int = 1) -> list[Slab]:
    """Contiguous slabs of whole unit cells (``unit`` rows), as even as the cells allow, with a
    halo of ``halo`` rows rounded up to whole cells. Every slab must own at least a halo's worth
    of rows, so that its halo comes from its neighbours alone."""
    if world < 1 or ny % unit:
        raise ValueError(f'{ny} rows do not split into whole unit cells of {unit} rows')
    cells = ny // unit
    if world > cells:
        raise ValueError(f'{world} ranks for {cells} unit-cell rows')
    h = -(-int(halo) // unit) * unit if world > 1 else 0
    out, start = [], 0
    for r in range(world):
        n = (cells // world + (1 if r < cells % world else 0)) * unit
        out.append(Slab(r, world, ny, nx, start, start + n, h, bool(pbc)))
        start += n
    if world > 1 and min(s.r1 - s.r0 for s in out) < h:
        raise ValueError(f'slabs of {min(s.r1 - s.r0 for s in out)} rows cannot hold a halo of {h} rows: use fewer ranks')
    return out


def exchange_halo(local, slab: Slab, group=None):
    """Fill the halo rows of ``local`` (a (rows, nx, ...) tensor laid out as ``slab.rows``) from
    the neighbouring ranks' owned rows, in place. Every rank calls it (collective)."""
    import torch.distributed as dist
    if slab.world == 1 or slab.h == 0:
        return local
    own = local[slab.own]
    n_own = own.shape[0]
    prev, nxt = (slab.rank - 1) % slab.world, (slab.rank + 1) % slab.world
    ops, recv = [], []
    has_prev = slab.pbc or slab.rank > 0
    has_next = slab.pbc or slab.rank < slab.world - 1
    # tag 0: rows travelling down to the previous rank (its upper halo); tag 1: up to the next
    if has_prev:
        ops.append(dist.P2POp(dist.isend, own[:slab.h].contiguous(), prev, group, tag=0))
        buf = local.new_empty(local[:slab.lo].shape)
        ops.append(dist.P2POp(dist.irecv, buf, prev, group, tag=1))
        recv.append((slice(0, slab.lo), buf))
    if has_next:
        ops.append(dist.P2POp(dist.isend, own[n_own - slab.h:].contiguous(), nxt, group, tag=1))
        buf = local.new_empty(local[slab.lo + n_own:].shape)
        ops.append(dist.P2POp(dist.irecv, buf, nxt, group, tag=0))
        recv.append((slice(slab.lo + n_own, slab.lo + n_own + slab.hi), buf))
    for w in dist.batch_isend_irecv(ops):
        w.wait()
    for sl, buf in recv:
        local[sl] = buf
    return local


def gather_switches(sw, group=None):
    """All ranks' switches of one step, merged into the single-process list order. ``sw``: an
    int64 tensor (k, 3) of (order key, global y, global x) on this rank, where the order key is
    the switch's position in the list one process would make (e.g. the candidate index of a
    Metropolis step). Returns the (K, 3) tensor sorted by order key, the same on every rank."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    k = torch.tensor([sw.shape[0]], dtype=torch.int64, device=sw.device)
    ks = [torch.zeros_like(k) for _ in range(world)]
    dist.all_gather(ks, k, group=group)
    most = int(max(int(x) for x in ks))
    pad = sw.new_zeros((most, 3))
    pad[:sw.shape[0]] = sw
    parts = [torch.zeros_like(pad) for _ in range(world)]
    dist.all_gather(parts, pad, group=group)
    allsw = torch.cat([p[:int(n)] for p, n in zip(parts, ks)])
    return allsw[torch.argsort(allsw[:, 0], stable=True)]


def slab_switches(allsw, slab: Slab, wy: int) -> np.ndarray:
    """The switches (global (order, y, x) rows, in list order) whose window of half-height
    ``wy`` reaches the slab's owned rows, as local (y, x) coordinates of the slab: the switch
    list of hs_dipolar_update on the slab's arrays. The halo of ``h >= wy`` rows guarantees each
    such switch lies inside the slab."""
    a = np.asarray(allsw.cpu() if hasattr(allsw, 'cpu') else allsw, dtype=np.int64).reshape(-1, 3)
    out = []
    for _, y, x in a:
        d = y - slab.r0
        if slab.pbc:
            d = (d + wy) % slab.ny - wy          # signed offset from r0, nearest image
        if -wy <= d < (slab.r1 - slab.r0) + wy:
            ly = slab.local_row(int(y))
            if ly is None:
                raise ValueError(f'switch row {y} reaches slab {slab.rank} but lies outside its halo')
            out.append((ly, int(x)))
    return np.asarray(out, dtype=np.int32).reshape(-1, 2)


def global_argmin(key: float, idx: int, group=None) -> tuple[float, int]:
    """The smallest (key, global row-major index) over the ranks, ties to the smaller index
    (numpy nanargmin); idx < 0 means the rank has no candidate."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    mine = torch.tensor([key if idx >= 0 else np.inf, float(idx)], dtype=torch.float64)
    parts = [torch.zeros_like(mine) for _ in range(world)]
    dist.all_gather(parts, mine, group=group)
    best = (np.inf, -1)
    for p in parts:
        k, i = float(p[0]), int(p[1])
        if i < 0:
            continue
        if best[1] < 0 or k < best[0] or (k == best[0] and i < best[1]):
            best = (k, i)
    return best
