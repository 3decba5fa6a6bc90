"""Lattice geometry for the oracle (test infrastructure, FP64, host only).

ORACLE module: only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it. It restates the geometry half of the reference's
``Magnets.__init__`` (hotspice/core.py:57-130) for the lattices the hot-path
workloads use, independently of the product's own geometry code.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class Geometry:
    nx: int
    ny: int
    dx: np.ndarray          # (nx,) spacing after each column, hotspice/core.py:382-392
    dy: np.ndarray          # (ny,)
    occupation: np.ndarray  # (ny, nx) int 0/1
    in_plane: bool
    nn_mask: np.ndarray     # nearest-neighbour mask (ASI._get_nearest_neighbors)
    orientation: np.ndarray | None = None  # (ny, nx, 2) for in-plane lattices
    angles: np.ndarray | None = None
    name: str = ''

    @property
    def x(self):
        x = np.zeros(self.nx); x[1:] = np.cumsum(self.dx)[:-1]; return x

    @property
    def y(self):
        y = np.zeros(self.ny); y[1:] = np.cumsum(self.dy)[:-1]; return y


def _tile_to(value, n):
    v = np.asarray(value, dtype=float).reshape(-1)
    return np.tile(v, math.ceil(n / v.size))[:n]


def _grids(nx, ny):
    ixx, iyy = np.meshgrid(np.arange(nx), np.arange(ny))
    return ixx, iyy


def _ip_orientation(angles_raw, occupation, extra_angle):
    """hotspice/core.py:182-193: angles * occupation, cos/sin masked by occupation."""
    angles = (angles_raw + extra_angle) * occupation
    o = np.zeros(occupation.shape + (2,))
    o[:, :, 0] = np.cos(angles) * occupation
    o[:, :, 1] = np.sin(angles) * occupation
    return o, angles


def oop_square(a, nx, ny=None):
    """hotspice/ASI.py:48-78."""
    ny = nx if ny is None else ny
    occ = np.ones((ny, nx), dtype=int)
    nn = np.array([[0, 1, 0], [1, 0, 1], [0, 1, 0]])
    return Geometry(nx, ny, _tile_to(a, nx), _tile_to(a, ny), occ, False, nn, name='OOP_Square')


def ip_square(a, nx, ny=None, angle=0.0):
    """hotspice/ASI.py:266-301 (IP_Square_Closed): spacing a/2, occupation (ix+iy)%2==1,
    angle pi/2 on odd rows."""
    ny = nx if ny is None else ny
    ixx, iyy = _grids(nx, ny)
    occ = ((ixx + iyy) % 2 == 1).astype(int)
    ang = np.zeros((ny, nx)); ang[iyy % 2 == 1] = math.pi / 2
    o, angles = _ip_orientation(ang, occ, angle)
    nn = np.array([[1, 0, 1], [0, 0, 0], [1, 0, 1]])
    return Geometry(nx, ny, _tile_to(a / 2, nx), _tile_to(a / 2, ny), occ, True, nn, o, angles, 'IP_Square')


def ip_pinwheel(a, nx, ny=None, angle=0.0):
    """hotspice/ASI.py:304-314,357: IP_Square rotated by -pi/4."""
    g = ip_square(a, nx, ny, angle=angle - math.pi / 4)
    g.name = 'IP_Pinwheel'
    return g


def ip_kagome(a, nx, ny=None, PBC=False, angle=0.0):
    """hotspice/ASI.py:371-402."""
    if ny is None:
        ny = int(nx / math.sqrt(3)) // 4 * 4
        if not PBC:
            ny -= 1
    ixx, iyy = _grids(nx, ny)
    occ = np.zeros((ny, nx), dtype=int)
    occ[(ixx + iyy) % 4 == 1] = 1
    occ[(ixx - iyy) % 4 == 3] = 1
    ang = np.ones((ny, nx)) * math.pi / 2
    ang[((ixx - iyy) % 4 == 1) & (ixx % 2 == 1)] = -math.pi / 6
    ang[((ixx + iyy) % 4 == 3) & (ixx % 2 == 1)] = math.pi / 6
    o, angles = _ip_orientation(ang, occ, angle)
    dx = a / 4
    nn = np.array([[0, 1, 0, 1, 0], [1, 0, 0, 0, 1], [0, 1, 0, 1, 0]])
    return Geometry(nx, ny, _tile_to(dx, nx), _tile_to(math.sqrt(3) * dx, ny), occ, True, nn, o, angles, 'IP_Kagome')


def _periodic(arr, px, py):
    """True if ``arr`` repeats with period px along axis 1 and py along axis 0
    (the property tested by hotspice/utils.py:42-66)."""
    H, W = arr.shape[:2]
    base = arr[:py, :px, ...]
    reps = (math.ceil(H / py), math.ceil(W / px)) + (1,) * (arr.ndim - 2)
    return np.allclose(np.tile(base, reps)[:H, :W, ...], arr)


def unitcell(g: Geometry, max_cell=100):
    """hotspice/core.py:146-161: smallest (ux, uy) in the same search order."""
    arr = g.orientation if g.in_plane else g.occupation
    dxr, dyr = g.dx.reshape(1, -1), g.dy.reshape(-1, 1)
    for n in range(1, min(g.nx + g.ny + 1, max_cell + 1)):
        for uy in range(max(0, n - g.nx) + 1, min(n, g.ny) + 1):
            ux = n - uy + 1
            if _periodic(arr, ux, uy) and _periodic(dxr, ux, 1) and _periodic(dyr, 1, uy):
                return ux, uy
    return g.nx, g.ny
