"""Lattice geometries (hotspice/ASI.py:15-535): occupation, angles, spacings, unit cells,
ground-state patterns and nearest-neighbour masks. Pure host-side geometry; the
simulation itself runs in :class:`hotspice_b200.core.Magnets`."""
from __future__ import annotations

import math

import numpy as np

from .core import Magnets


class OOP_ASI(Magnets):
    """Generic out-of-plane ASI."""

    def _get_angles(self):
        return np.nan * np.zeros_like(self.ixx, dtype=float)

    def correlation_NN(self, NN=None):
        """<S_i S_j> over nearest neighbours (hotspice/ASI.py:28-36)."""
        from scipy import signal  # host-side observable, not on the hot path
        if NN is None:
            NN = self._get_nearest_neighbors()
        b = 'wrap' if self.PBC else 'fill'
        m = self.m.cpu().numpy()
        total = signal.convolve2d(self.occupation, NN, mode='same', boundary=b) * self.occupation
        s = signal.convolve2d(m, NN, mode='same', boundary=b)
        v = np.where(total != 0)
        return float(np.mean(m[v] * s[v] / total[v]))


class IP_ASI(Magnets):
    """Generic in-plane ASI."""


def _n(nx, ny, n):
    nx = n if nx is None else nx
    ny = n if ny is None else ny
    if nx is None or ny is None:
        raise AttributeError("Must specify <n> if either <nx> or <ny> are not specified.")
    return nx, ny


class OOP_Square(OOP_ASI):
    def __init__(self, a: float, n: int = None, *, nx: int = None, ny: int = None, **kwargs):
        self.a = a
        nx, ny = _n(nx, ny, n)
        dx, dy = kwargs.pop('dx', a), kwargs.pop('dy', a)
        super().__init__(nx, ny, dx, dy, in_plane=False, **kwargs)

    def _set_m(self, pattern: str):
        if str(pattern).strip().lower() == 'afm':
            return ((self.ixx - self.iyy) % 2) * 2 - 1
        return super()._set_m(pattern)

    def _get_occupation(self):
        return np.ones_like(self.ixx)

    def _get_appropriate_avg(self):
        return ['point', 'square', 'crossfour']

    def _get_AFMmask(self):
        return np.array([[0, -1], [-1, 2]], dtype='float') / 4

    def _get_nearest_neighbors(self):
        return np.array([[0, 1, 0], [1, 0, 1], [0, 1, 0]])

    def _get_groundstate(self):
        return 'afm'

    def correlation_NN(self, N=1):
        NN = {1: None, 2: np.array([[1, 0, 1], [0, 0, 0], [1, 0, 1]]),
              3: np.array([[0, 0, 1, 0, 0], [0, 0, 0, 0, 0], [1, 0, 0, 0, 1], [0, 0, 0, 0, 0], [0, 0, 1, 0, 0]])}[N]
        return super().correlation_NN(NN=NN)


class OOP_Triangle(OOP_ASI):
    def __init__(self, a: float, n: int = None, *, nx: int = None, ny: int = None, **kwargs):
        self.a = a
        if nx is None:
            nx = n
        if ny is None:
            ny = int(nx / math.sqrt(3)) // 2 * 2
            if not kwargs.get('PBC', False):
                ny -= 1
        dx = kwargs.pop('dx', a / 2)
        dy = kwargs.pop('dy', math.sqrt(3) * dx)
        super().__init__(nx, ny, dx, dy, in_plane=False, **kwargs)

    def _set_m(self, pattern: str):
        if str(pattern).strip().lower() == 'afm':
            return ((self.ixx - self.iyy) // 2 % 2) * 2 - 1
        return super()._set_m(pattern)

    def _get_occupation(self):
        return (self.ixx + self.iyy) % 2 == 1

    def _get_nearest_neighbors(self):
        return np.array([[0, 1, 0, 1, 0], [1, 0, 0, 0, 1], [0, 1, 0, 1, 0]])

    def _get_groundstate(self):
        return 'afm'


class OOP_Honeycomb(OOP_ASI):
    def __init__(self, a: float, n: int = None, *, nx: int = None, ny: int = None, **kwargs):
        self.a = a
        if nx is None:
            nx = n
        if ny is None:
            ny = int(nx / math.sqrt(3)) // 2 * 2
            if not kwargs.get('PBC', False):
                ny -= 1
        dy = kwargs.pop('dx', a / 2)
        dx = kwargs.pop('dy', math.sqrt(3) * dy)
        super().__init__(nx, ny, dx, dy, in_plane=False, **kwargs)

    def _set_m(self, pattern: str):
        if str(pattern).strip().lower() == 'afm':
            return (self.iyy % 3 == 1) * 2 - 1
        return super()._set_m(pattern)

    def _get_occupation(self):
        occ = np.ones_like(self.ixx)
        occ[(self.ixx + self.iyy) % 2 == 0] = 0
        occ[self.iyy % 3 == 2] = 0
        return occ

    def _get_nearest_neighbors(self):
        return np.array([[0, 1, 0, 1, 0], [1, 0, 0, 0, 1], [0, 1, 0, 1, 0]])

    def _get_groundstate(self):
        return 'afm'


class IP_Ising(IP_ASI):
    def __init__(self, a: float, n: int = None, *, nx: int = None, ny: int = None, **kwargs):
        self.a = a
        nx, ny = _n(nx, ny, n)
        dx, dy = kwargs.pop('dx', a), kwargs.pop('dy', a)
        super().__init__(nx, ny, dx, dy, in_plane=True, **kwargs)

    def _set_m(self, pattern: str):
        if str(pattern).strip().lower() == 'afm':
            return (self.iyy % 2) * 2 - 1
        return super()._set_m(pattern)

    def _get_angles(self):
        return np.zeros_like(self.ixx, dtype=float)

    def _get_occupation(self):
        return np.ones_like(self.ixx)

    def _get_nearest_neighbors(self):
        return np.array([[0, 1, 0], [1, 0, 1], [0, 1, 0]])

    def _get_groundstate(self):
        return 'uniform'


class IP_Square_Closed(IP_ASI):
    def __init__(self, a: float, n: int = None, *, nx: int = None, ny: int = None, **kwargs):
        self.a = a
        nx, ny = _n(nx, ny, n)
        dx, dy = kwargs.pop('dx', a / 2), kwargs.pop('dy', a / 2)
        super().__init__(nx, ny, dx, dy, in_plane=True, **kwargs)

    def _set_m(self, pattern: str):
        if str(pattern).strip().lower() == 'afm':
            return ((self.ixx - self.iyy) // 2 % 2) * 2 - 1
        return super()._set_m(pattern)

    def _get_angles(self):
        angles = np.zeros_like(self.ixx, dtype=float)
        angles[self.iyy % 2 == 1] = math.pi / 2
        return angles

    def _get_occupation(self):
        return (self.ixx + self.iyy) % 2 == 1

    def _get_appropriate_avg(self):
        return ['cross', 'square', 'squarefour']

    def _get_nearest_neighbors(self):
        return np.array([[1, 0, 1], [0, 0, 0], [1, 0, 1]])

    def _get_groundstate(self):
        return 'afm'


class IP_Pinwheel_Diamond(IP_Square_Closed):
    def __init__(self, a: float, n: int = None, *, nx: int = None, ny: int = None, **kwargs):
        kwargs['angle'] = kwargs.get('angle', 0) - math.pi / 4
        super().__init__(a, n=n, nx=nx, ny=ny, **kwargs)

    def _get_appropriate_avg(self):
        return ['squarefour', 'cross']

    def _get_groundstate(self):
        return 'uniform' if self.PBC else 'vortex'


class IP_Square(IP_Square_Closed):
    pass


def count_square_vertices(mm: Magnets, counts: bool = False):
    """Vertex-type fractions (N1, N2, N3, N4) of an in-plane square ASI state, counted on the
    device (hs_square_vertex_counts): the counterpart of count_square_vertices in
    examples/IP_SquareVertices.py:19-35. Vertices are the cells with even x and y; their four
    magnets are the neighbours with periodic wrap. Type 1 is the flower state, 3 and 4 have two
    and four magnets pointing in, 2 is the rest. Like the reference, the fractions require every
    vertex to be of one of the four types (an odd lattice side wraps a vertex cell in as a
    neighbour, which the reference's assertion refuses too). ``counts=True`` returns the four
    integer counts as they are, without that check."""
    import torch
    from . import _lib
    out = torch.empty(4, dtype=torch.int64, device=mm.device)
    _lib.check(_lib.load().hs_square_vertex_counts(mm._m_dev.data_ptr(), mm.nx, mm.ny, out.data_ptr(), mm._stream()),
               'hs_square_vertex_counts')
    c = out.cpu().numpy()
    if counts:
        return tuple(int(v) for v in c)
    total = int(c.sum())
    if total != ((mm.nx + 1) // 2) * ((mm.ny + 1) // 2):
        raise RuntimeError(f'vertex counts {c.tolist()} do not add up to the number of vertices')
    return tuple(float(v) / total for v in c)


class IP_Pinwheel(IP_Pinwheel_Diamond):
    pass


class IP_Square_Open(IP_ASI):
    def __init__(self, a: float, n: int = None, *, nx: int = None, ny: int = None, **kwargs):
        self.a = a
        nx, ny = _n(nx, ny, n)
        dx, dy = kwargs.pop('dx', a / math.sqrt(2)), kwargs.pop('dy', a / math.sqrt(2))
        super().__init__(nx, ny, dx, dy, in_plane=True, **kwargs)

    def _set_m(self, pattern: str):
        if str(pattern).strip().lower() == 'afm':
            return (self.iyy % 2) * 2 - 1
        return super()._set_m(pattern)

    def _get_angles(self):
        angles = -np.ones_like(self.ixx, dtype=float) * math.pi / 4
        angles[(self.iyy + self.ixx) % 2 == 1] = math.pi / 4
        return angles

    def _get_occupation(self):
        return np.ones_like(self.ixx)

    def _get_nearest_neighbors(self):
        return np.array([[0, 1, 0], [1, 0, 1], [0, 1, 0]])

    def _get_groundstate(self):
        return 'afm'


class IP_Pinwheel_LuckyKnot(IP_Square_Open):
    def __init__(self, a: float, n: int = None, *, nx: int = None, ny: int = None, **kwargs):
        kwargs['angle'] = kwargs.get('angle', 0) - math.pi / 4
        super().__init__(a, n=n, nx=nx, ny=ny, **kwargs)

    def _get_groundstate(self):
        return 'uniform' if self.PBC else 'vortex'


class IP_Kagome(IP_ASI):
    def __init__(self, a: float, n: int = None, *, nx: int = None, ny: int = None, **kwargs):
        self.a = a
        if nx is None:
            nx = n
        if ny is None:
            ny = int(nx / math.sqrt(3)) // 4 * 4
            if not kwargs.get('PBC', False):
                ny -= 1
        dx = kwargs.pop('dx', a / 4)
        dy = kwargs.pop('dy', math.sqrt(3) * dx)
        super().__init__(nx, ny, dx, dy, in_plane=True, **kwargs)

    def _set_m(self, pattern: str):
        if str(pattern).strip().lower() == 'afm':
            m = np.ones_like(self.ixx)
            m[(self.ixx + self.iyy) % 4 == 3] *= -1
            return m
        return super()._set_m(pattern)

    def _get_angles(self):
        angles = np.ones_like(self.ixx, dtype=float) * math.pi / 2
        angles[((self.ixx - self.iyy) % 4 == 1) & (self.ixx % 2 == 1)] = -math.pi / 6
        angles[((self.ixx + self.iyy) % 4 == 3) & (self.ixx % 2 == 1)] = math.pi / 6
        return angles

    def _get_occupation(self):
        occ = np.zeros_like(self.ixx)
        occ[(self.ixx + self.iyy) % 4 == 1] = 1
        occ[(self.ixx - self.iyy) % 4 == 3] = 1
        return occ

    def _get_appropriate_avg(self):
        return ['cross', 'point', 'triangle', 'hexagon']

    def _get_nearest_neighbors(self):
        return np.array([[0, 1, 0, 1, 0], [1, 0, 0, 0, 1], [0, 1, 0, 1, 0]])

    def _get_groundstate(self):
        return 'uniform'


class IP_Triangle(IP_Kagome):
    def __init__(self, a: float, n: int = None, *, nx: int = None, ny: int = None, **kwargs):
        kwargs['angle'] = kwargs.get('angle', 0) - math.pi / 2
        super().__init__(a, n=n, nx=nx, ny=ny, **kwargs)

    def _get_groundstate(self):
        return 'afm'
