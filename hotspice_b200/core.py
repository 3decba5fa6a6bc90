"""Magnets / SimParams / Scheme with the reference API (hotspice/core.py:29-1006), running the
kinetic Monte Carlo hot path on the sm_100a kernels of libhotspice_sm100.so.

Geometry, kernels and parameter fields are prepared on the host in FP64 (as the reference
does); the simulation state (spins, energies, counters, simulated time) lives on the GPU.
``update()`` is the plain, one-step-per-call form (it returns the switched indices and so
synchronises once per call). ``progress()`` runs whole chunks of steps on the device, with
the stopping rule of hotspice/core.py:753-760 evaluated by the kernels, replayed from
captured CUDA graphs, and synchronises only once per chunk.

All random variates come from the Philox4x32-10 stream keyed by ``seed`` (one stream call
per vectorised reference draw, see include/hotspice_b200.h), so a run is reproducible and
comparable draw-for-draw with the reference fed the same stream.
"""
from __future__ import annotations

import ctypes
import math
import os
import warnings
from abc import ABC
from dataclasses import dataclass, field
from enum import Enum, auto
from functools import lru_cache
from textwrap import dedent
from typing import Literal

import numpy as np
import torch

from . import _lib, config
from .energies import DiMonopolarEnergy, DipolarEnergy, Energy, ExchangeEnergy, ZeemanEnergy
from .utils import as_2D_array, check_repetition, copy_to_device, full_obj_name, lower_than, to_device

__all__ = ['kB', 'SimParams', 'Magnets', 'Scheme', 'EngineConfig', 'Unitcell']

kB = 1.380649e-23


class Scheme(Enum):
    NEEL = auto()
    METROPOLIS = auto()
    WOLFF = auto()


@dataclass(slots=True)
class SimParams:
    """hotspice/core.py:34-53 (same fields, defaults and validation)."""
    SIMULTANEOUS_SWITCHES_CONVOLUTION_OR_SUM_CUTOFF: int = 20
    REDUCED_KERNEL_SIZE: int = 20
    UPDATE_SCHEME: Scheme | str = Scheme.NEEL
    MULTISAMPLING_SCHEME: Literal['single', 'grid', 'Poisson', 'cluster'] = 'grid'
    ENERGY_BARRIER_METHOD: Literal['simple', 'parabolic'] = 'simple'
    METROPOLIS_TIME: bool = False

    def __post_init__(self):
        self.SIMULTANEOUS_SWITCHES_CONVOLUTION_OR_SUM_CUTOFF = int(self.SIMULTANEOUS_SWITCHES_CONVOLUTION_OR_SUM_CUTOFF)
        self.REDUCED_KERNEL_SIZE = int(self.REDUCED_KERNEL_SIZE)
        if not isinstance(self.UPDATE_SCHEME, Scheme):
            allowed = {'Néel': Scheme.NEEL, 'Neel': Scheme.NEEL, 'Metropolis': Scheme.METROPOLIS,
                       'Glauber': Scheme.METROPOLIS, 'Wolff': Scheme.WOLFF}
            if self.UPDATE_SCHEME not in allowed.keys():
                raise ValueError(f"UPDATE_SCHEME='{self.UPDATE_SCHEME}' is invalid: allowed values are {allowed.keys()}.")
            self.UPDATE_SCHEME = allowed[self.UPDATE_SCHEME]
        if self.MULTISAMPLING_SCHEME not in (allowed := ['single', 'grid', 'Poisson', 'cluster']):
            raise ValueError(f"MULTISAMPLING_SCHEME='{self.MULTISAMPLING_SCHEME}' is invalid: allowed values are {allowed}.")


@dataclass
class EngineConfig:
    """Engine knobs that are not part of the reference's SimParams."""
    resync_every: int = 0          # full dipolar recompute every N progress() steps (0: never)
    recompute: str = 'auto'        # 'auto' | 'direct64' | 'direct32' | 'igemm'
    direct_max_pairs: float = 4e11 # 'auto' uses the FP64 direct sum up to this many (cell, window) pairs
    persistent: bool = True        # run()/progress() as one persistent cluster launch (hs_engine_run)
    cluster_size: int = 0          # CTAs per cluster for the persistent launch (0: cost model)
    use_graphs: bool = True        # otherwise: replay progress() chunks from captured CUDA graphs
    graph_steps: int = 64          # steps per captured chunk
    igemm_splits: int = 3          # BF16 terms of the split kernel in the implicit GEMM (2: faster, ~1e-6 rel)


@dataclass(slots=True)
class Unitcell:
    x: int
    y: int


@dataclass
class History:
    E: list = field(default_factory=list)
    T: list = field(default_factory=list)
    t: list = field(default_factory=list)
    m: list = field(default_factory=list)

    def entry(self, mm: 'Magnets'):
        self.E.append(mm.E_tot)
        self.T.append(mm.T_avg)
        self.t.append(mm.t if mm.t != 0 else mm.switches)
        self.m.append(mm.m_avg)

    def clear(self):
        self.E.clear(); self.T.clear(); self.t.clear(); self.m.clear()


def check_progress_limits(t_max, MCsteps_max):
    """progress() stops when either limit is reached (hotspice/core.py:753-760); with both
    infinite it would run forever, so that is refused."""
    if not (float(t_max) < math.inf or float(MCsteps_max) < math.inf):
        raise ValueError('progress() needs a finite t_max or MCsteps_max: with both infinite it never ends')


def _ptr(t):
    return None if t is None else t.data_ptr()


class RunSummary:
    """What Magnets.summary_async copied out: pinned host buffers filled by the stream,
    readable once the event has completed."""

    def __init__(self, mm, host, divs, event):
        self._mm, self._host, self._divs, self.event = mm, host, divs, event

    def ready(self) -> bool:
        return self.event.query()

    def result(self) -> dict:
        """counters (record), E_tot, m_avg and state (int8 spins or None); raises when an
        enqueued recompute reported a status, like Magnets.check_resync."""
        self.event.synchronize()
        h = self._host
        if 'status' in h:
            for st in h['status'].tolist():
                if st:
                    raise RuntimeError(f'hs_dipolar_full_igemm reported status {st} '
                                       f'(1: wait timed out, 2: moment not uniform)')
        vals = h['scal'].tolist()
        ne = len(self._divs)
        rec = np.frombuffer(h['counters'].numpy().tobytes(), dtype=_lib.COUNTERS_DTYPE)[0]
        return dict(counters=rec, E_tot=float(sum(v / d for v, d in zip(vals[:ne], self._divs))),
                    m_avg=self._mm._m_avg_from(vals[ne:]),
                    state=h['state'].numpy().copy() if 'state' in h else None)


class Magnets(ABC):
    """hotspice/core.py:56-980. See the module docstring for what runs where."""

    def __init__(self, nx: int, ny: int, dx, dy, *, T=300, E_B=0., moment=None, Msat=800e3, V=2e-22,
                 pattern=None, energies=None, PBC: bool = False, m_perp_factor: float = None, E_B_std: float = None,
                 major_axis: float = 0, minor_axis: float = None, angle: float = 0., params: SimParams = None,
                 in_plane: bool = False, seed: int | None = None, engine: EngineConfig | None = None,
                 device=None):
        if not torch.cuda.is_available():
            raise RuntimeError('hotspice_b200 runs on a CUDA device (sm_100a); none is available')
        self._lib = _lib.load()
        if device is None:
            device = torch.device('cuda', config.DEVICE_ID if config.DEVICE_ID is not None else torch.cuda.current_device())
        self.device = torch.device(device)
        self.params = SimParams() if params is None else params
        self.engine = EngineConfig() if engine is None else engine
        self.seed = int.from_bytes(os.urandom(8), 'little') if seed is None else int(seed) & (2 ** 64 - 1)
        self._energies: list[Energy] = []
        self._version = 0
        self._L = None
        self._graphs = {}
        self._plans = {}
        self._scratch = {}
        self.in_plane = in_plane
        self.nx, self.ny = int(nx), int(ny)
        self.ixx, self.iyy = np.meshgrid(np.arange(self.nx), np.arange(self.ny))
        self._dx_set(dx)
        self._dy_set(dy)
        self.occupation = self._get_occupation().astype(bool).astype(int)
        with np.errstate(invalid='ignore', divide='ignore'):
            self._occupation_inf = 1 / self.occupation
        self.nonzero = np.nonzero(self.occupation)
        self._nonzero_array = np.asarray(self.nonzero).reshape(2, -1)
        self.n = int(np.sum(self.occupation))
        if self.n == 0:
            raise ValueError(f"Can not initialize {full_obj_name(self)} of size {self.nx}x{self.ny}, as this does not contain any spins.")
        if self.in_plane:
            self._initialize_ip(angle=angle)
        self.unitcell = self._get_unitcell()
        self._PBC = False
        self.PBC = PBC
        # device state
        dev = self.device
        self._occ_dev = to_device(self.occupation, dev, torch.int8)
        self._nonzero_dev = to_device(np.flatnonzero(self.occupation), dev, torch.int32)
        self._m_dev = torch.zeros((self.ny, self.nx), device=dev, dtype=torch.int8)
        self._mm_dev = torch.zeros((self.ny, self.nx), device=dev, dtype=torch.float32)
        self._counters = torch.zeros(ctypes.sizeof(_lib.HsCounters), device=dev, dtype=torch.uint8)
        self._orient_dev = to_device(self.orientation, dev, torch.float32) if self.in_plane else None
        self._moment_np = np.ones((self.ny, self.nx))
        self._mom_dev = torch.ones((self.ny, self.nx), device=dev, dtype=torch.float32)
        self.initialize_m(self._get_groundstate() if pattern is None else pattern, update_energy=False)
        self.T = T
        self.E_B = E_B
        if E_B_std is not None:
            g = np.random.Generator(np.random.PCG64(self.seed))
            self.E_B = self._EB_np * g.normal(1, E_B_std, size=self._EB_np.shape)
        self.moment = Msat * V if moment is None else moment
        self._m_perp_factor = 0.0
        self.m_perp_factor = in_plane if m_perp_factor is None else m_perp_factor
        self.major_axis = major_axis
        self.minor_axis = major_axis if minor_axis is None else minor_axis
        self.history = History()
        if energies is None:
            energies = (DipolarEnergy(),)
        elif isinstance(energies, Energy):
            energies = (energies,)
        else:
            energies = tuple(energies)
        for energy in energies:
            self.add_energy(energy)

    # ------------------------------------------------------------------ geometry (host)
    def _dx_set(self, value):
        value = np.asarray(value, dtype=float).reshape(-1)
        self._dx = np.tile(value, math.ceil(self.nx / value.size))[:self.nx]
        self.x = np.zeros(self.nx)
        self.x[1:] = np.cumsum(self._dx)[:-1]
        self.xx, _ = np.meshgrid(self.x, np.empty(self.ny))
        self.x_min, self.x_max = float(self.x[0]), float(self.x[-1])

    def _dy_set(self, value):
        value = np.asarray(value, dtype=float).reshape(-1)
        self._dy = np.tile(value, math.ceil(self.ny / value.size))[:self.ny]
        self.y = np.zeros(self.ny)
        self.y[1:] = np.cumsum(self._dy)[:-1]
        _, self.yy = np.meshgrid(np.empty(self.nx), self.y)
        self.y_min, self.y_max = float(self.y[0]), float(self.y[-1])

    @property
    def dx(self):
        return self._dx

    @dx.setter
    def dx(self, value):
        self._dx_set(value)
        self._reinit_energies()

    @property
    def dy(self):
        return self._dy

    @dy.setter
    def dy(self, value):
        self._dy_set(value)
        self._reinit_energies()

    def _initialize_ip(self, angle: float = 0.):
        """hotspice/core.py:182-193."""
        self.original_angles = self._get_angles() + angle
        self.angles = self.original_angles * self.occupation
        self.orientation = np.zeros(self.ixx.shape + (2,))
        self.orientation[:, :, 0] = np.cos(self.angles) * self.occupation
        self.orientation[:, :, 1] = np.sin(self.angles) * self.occupation

    def _get_unitcell(self, max_cell=100):
        """hotspice/core.py:146-161."""
        dx, dy = self.dx.reshape(1, -1), self.dy.reshape(-1, 1)
        for n in range(1, min(self.nx + self.ny + 1, max_cell + 1)):
            for uy in range(max(0, n - self.nx) + 1, min(n, self.ny) + 1):
                ux = n - uy + 1
                if check_repetition(self.orientation if self.in_plane else self.occupation, ux, uy):
                    if check_repetition(dx, ux, 1) and check_repetition(dy, 1, uy):
                        return Unitcell(ux, uy)
        warnings.warn(dedent(f"""
            Could not detect a reasonably sized unit cell. Defaulting to entire domain {self.nx}x{self.ny}."""), stacklevel=2)
        return Unitcell(self.nx, self.ny)

    def _get_closest_dist(self):
        sl = np.where(self.occupation[:self.unitcell.y * 2, :self.unitcell.x * 2])
        pos = np.asarray([self.xx[sl], self.yy[sl]]).T
        d = np.sqrt(((pos[:, None, :] - pos[None, :, :]) ** 2).sum(-1))
        return float(d[np.triu_indices(len(pos), 1)].min())

    @property
    def shape(self):
        return (self.ny, self.nx)

    @property
    def PBC(self):
        return self._PBC

    @PBC.setter
    def PBC(self, value: bool):
        if hasattr(self, 'unitcell') and value and (self.nx % self.unitcell.x != 0 or self.ny % self.unitcell.y != 0):
            warnings.warn(dedent(f"""
                WARNING: PBC can not be enabled, because there is a non-integer number of unit cells along the x- and/or y-axis,
                         so the boundaries do not match (unit cell has size {self.unitcell.x}x{self.unitcell.y})."""), stacklevel=2)
            self._PBC = False
            return
        self._PBC = bool(value)
        self._reinit_energies()

    def _reinit_energies(self):
        for energy in getattr(self, '_energies', []):
            energy.initialize(self)
        if hasattr(self, '_version'):
            self._state_changed()

    # ------------------------------------------------------------------ state
    def _state_changed(self):
        self._version += 1
        self._L = None
        self._graphs.clear()

    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def _field(self, value):
        return as_2D_array(value, self.shape)

    @property
    def m(self) -> torch.Tensor:
        """Spins as a float64 tensor (-1, 0, +1). Assign to ``m`` (or call initialize_m) to
        change them; the returned tensor is a copy."""
        return self._m_dev.double()

    @m.setter
    def m(self, value):
        self._set_m_array(as_2D_array(value, self.shape))

    def _set_m_array(self, arr):
        arr = np.sign(np.asarray(arr, dtype=float))
        copy_to_device(self._m_dev, arr)
        self._mm_dev.copy_(self._m_dev.float() * self._mom_dev)

    def initialize_m(self, pattern='random', *, angle: float = 0, update_energy: bool = True):
        """hotspice/core.py:163-180."""
        if isinstance(pattern, str):
            m = self._set_m(pattern)
        else:
            try:
                m = as_2D_array(pattern, self.shape)
            except (ValueError, TypeError):
                raise ValueError("Argument <pattern> could not be parsed as a valid array for <self.m>.")
        m = np.sign(np.asarray(m, dtype=float)) * self.occupation
        flip = self._get_m_uniform() != self._get_m_uniform(angle)
        m[flip] *= -1
        self._set_m_array(m)
        if update_energy:
            self.update_energy()

    def _get_m_uniform(self, angle=0):
        angle += 1e-6
        if self.in_plane:
            return self.occupation * (2 * ((self.orientation[:, :, 0] * np.cos(angle) + self.orientation[:, :, 1] * np.sin(angle)) >= 0) - 1)
        return np.ones_like(self.xx) * ((np.floor(angle / math.pi - .5) % 2) * 2 - 1)

    def _random_pm1(self):
        """rng.integers(0, 2, size) * 2 - 1 (hotspice/core.py:951) from the Philox stream."""
        n = self.nx * self.ny
        u = torch.empty(n, device=self.device, dtype=torch.float64)
        call = int(self._read_counters()['rng_call'])
        _lib.check(self._lib.hs_philox_uniform(self.seed, call, n, u.data_ptr(), self._stream()), 'hs_philox_uniform')
        self._write_counters(rng_call=call + 1)
        return (torch.floor(u * 2) * 2 - 1).reshape(self.shape).cpu().numpy()

    def _set_m(self, pattern: str):
        """hotspice/core.py:924-952 (common patterns); subclasses add 'afm' etc."""
        match str(pattern).strip().lower():
            case 'uniform':
                return self._get_m_uniform()
            case 'vortex':
                m = np.ones_like(self.xx)
                if self.in_plane:
                    dxv = self.xx - (self.x_max - self.x_min) / 2
                    dyv = self.yy - (self.y_max - self.y_min) / 2
                    desired = (dxv + 1j * dyv) * (-1j + 1e-6)
                    dot = desired.real * self.orientation[:, :, 0] + desired.imag * self.orientation[:, :, 1]
                    dot[dot == 0] = 1
                    occ = np.where(self.occupation == 1)
                    m[occ] = np.sign(dot)[occ]
                else:
                    m[np.where(self.xx >= (self.x_max - self.x_min) / 2)] *= -1
                return m
            case str(unknown):
                if unknown != 'random':
                    warnings.warn(f"Pattern '{unknown}'' not recognized, defaulting to 'random'.", stacklevel=2)
                return self._random_pm1()

    # fields ------------------------------------------------------------------------
    @property
    def T(self):
        return torch.as_tensor(self._T_np, device=self.device)

    @T.setter
    def T(self, value):
        self._T_np = as_2D_array(value, self.shape)
        self.kBT = kB * self._T_np
        with np.errstate(divide='ignore'):
            self.beta = 1 / self.kBT
        self._T_zero = bool(np.any(self._T_np == 0))
        occ = self.occupation.astype(bool)
        bu = self.beta[occ] if occ.any() else self.beta.reshape(-1)
        self._beta_uniform = float(bu[0]) if (np.all(bu == bu[0]) and np.isfinite(bu[0])) else 0.0
        b = np.where(np.isfinite(self.beta), self.beta, 0.0)
        self._beta_dev = to_device(b, self.device, torch.float32)
        if hasattr(self, '_version'):
            self._state_changed()

    def set_T(self, f, /, *, center=False, crystalunits=False):
        xx = self.ixx if crystalunits else self.xx
        yy = self.iyy if crystalunits else self.yy
        lx = self.nx - 1 if crystalunits else self.x_max - self.x_min
        ly = self.ny - 1 if crystalunits else self.y_max - self.y_min
        self.T = f(xx - center * lx / 2, yy - center * ly / 2)

    @property
    def E_B(self):
        return torch.as_tensor(self._EB_np, device=self.device)

    @E_B.setter
    def E_B(self, value):
        self._EB_np = as_2D_array(value, self.shape)
        self._EB_dev = to_device(self._EB_np, self.device, torch.float32)
        self._state_changed()

    @property
    def moment(self):
        return torch.as_tensor(self._moment_np, device=self.device)

    @moment.setter
    def moment(self, value):
        self._moment_np = as_2D_array(value, self.shape)
        self._momentSq = self._moment_np * self._moment_np
        self._mom_dev = to_device(self._moment_np, self.device, torch.float32)
        self._mm_dev.copy_(self._m_dev.float() * self._mom_dev)
        for e in self._energies:
            if isinstance(e, ZeemanEnergy):
                e.set_field()
            elif isinstance(e, DiMonopolarEnergy):
                e._moment_changed()
        self._state_changed()

    @property
    def USE_PERP_ENERGY(self):
        return bool(self.m_perp_factor) and self.in_plane

    @property
    def m_perp_factor(self):
        return self._m_perp_factor

    @m_perp_factor.setter
    def m_perp_factor(self, value):
        if not isinstance(value, (int, float, bool)):
            raise ValueError("m_perp_factor must be scalar. It is not currently supported as a 2D array.")
        if value and not self.in_plane:
            warnings.warn("You set a nonzero `m_perp_energy`, but this has no effect for an OOP ASI.")
        used = self.USE_PERP_ENERGY
        self._m_perp_factor = float(value)
        self._state_changed()
        if not used and self.USE_PERP_ENERGY and self._energies:
            self.update_energy()

    # counters -----------------------------------------------------------------------
    def _read_counters(self):
        raw = self._counters.cpu().numpy()
        return np.frombuffer(raw.tobytes(), dtype=_lib.COUNTERS_DTYPE)[0]

    def _write_counters(self, **fields):
        rec = np.frombuffer(self._counters.cpu().numpy().tobytes(), dtype=_lib.COUNTERS_DTYPE).copy()
        for k, v in fields.items():
            rec[0][k] = v
        self._counters.copy_(torch.from_numpy(rec.view(np.uint8).copy()))
        self._ctl = None

    def _set_control(self, **fields):
        """Asynchronously set counter fields (no host synchronisation): each value goes
        through its own pinned staging buffer, ordered on the current stream."""
        ctl = getattr(self, '_ctl', None) or {}
        for k, v in fields.items():
            if ctl.get(k) == v:
                continue
            dt = _lib.COUNTERS_DTYPE.fields[k][0]
            off = _lib.COUNTERS_DTYPE.fields[k][1]
            b = torch.from_numpy(np.array([v], dtype=dt).view(np.uint8)).pin_memory()
            self._counters[off:off + b.numel()].copy_(b, non_blocking=True)
            ctl[k] = v
        self._ctl = ctl

    @property
    def t(self) -> float:
        return float(self._read_counters()['t'])

    @t.setter
    def t(self, value):
        self._write_counters(t=float(value))

    @property
    def switches(self) -> int:
        return int(self._read_counters()['switches'])

    @switches.setter
    def switches(self, value):
        self._write_counters(switches=int(value))

    @property
    def attempted_switches(self) -> int:
        return int(self._read_counters()['attempted'])

    @attempted_switches.setter
    def attempted_switches(self, value):
        self._write_counters(attempted=int(value))

    @property
    def MCsteps(self):
        return self.attempted_switches / self.n

    def reset_stats(self):
        self._write_counters(t=0.0, switches=0, attempted=0)

    @property
    def status(self) -> int:
        """Device status bits (HS_ST_*): bounded loops that gave up, capacity overflows."""
        return int(self._read_counters()['status'])

    @property
    def near_threshold(self) -> int:
        """Metropolis decisions whose margin |u - p| was within a 1e-6 relative energy change."""
        return int(self._read_counters()['near_threshold'])

    # energies -----------------------------------------------------------------------
    def add_energy(self, energy: Energy, exist_ok=False, verbose=True):
        if isinstance(energy, DipolarEnergy) and any(isinstance(e, DipolarEnergy) and type(e) is not type(energy)
                                                     for e in self._energies):
            raise NotImplementedError('the sm_100a path holds one magnetostatic kernel per lattice: '
                                      'DipolarEnergy and DiMonopolarEnergy cannot be combined')
        energy.initialize(self)
        for i, e in enumerate(self._energies):
            if type(e) is type(energy):
                if exist_ok:
                    return e
                if verbose:
                    warnings.warn(f"An instance of {type(energy).__name__} was already included in the simulation, and has now been overwritten.", stacklevel=2)
                self._energies[i] = energy
                self._state_changed()
                return
        self._energies.append(energy)
        self._state_changed()
        return energy

    def remove_energy(self, name: str, verbose=True):
        name = name.lower().replace('energy', '')
        for i, e in enumerate(self._energies):
            if name == e.shortname:
                self._energies.pop(i)
                self._state_changed()
                return
        if verbose:
            warnings.warn(f"There is no '{name}' energy associated with this Magnets object.", stacklevel=2)

    def has_energy(self, name: str):
        name = name.lower().replace('energy', '')
        return any(name == e.shortname for e in self._energies)

    def get_energy(self, name: str, verbose=True):
        name = name.lower().replace('energy', '')
        for e in self._energies:
            if name == e.shortname:
                return e
        if verbose:
            warnings.warn(f"There is no '{name}' energy associated with this Magnets object. Valid energies are: {[e.shortname for e in self._energies]}", stacklevel=2)
        return None

    def update_energy(self, index=None):
        """hotspice/core.py:241-253."""
        for energy in self._energies:
            if index is None:
                energy.update()
            else:
                idx = np.asarray(index).reshape(2, -1)
                if idx[0].size == 1:
                    energy.update_single(idx)
                elif idx[0].size > 1:
                    energy.update_multiple(idx)

    def switch_energy(self, indices2D=None):
        return sum(e.energy_switch(indices2D) for e in self._energies)

    def perp_energy(self, indices2D=None):
        if not self.USE_PERP_ENERGY:
            z = torch.zeros(self.shape, device=self.device, dtype=torch.float64)
            return z if indices2D is None else torch.zeros(np.asarray(indices2D).shape[1], device=self.device, dtype=torch.float64)
        tot = sum(e.E_perp for e in self._energies) * self.m_perp_factor
        if indices2D is None:
            return tot
        idx = torch.as_tensor(np.asarray(indices2D), device=self.device, dtype=torch.long)
        return tot[idx[0], idx[1]]

    @property
    def E(self):
        return sum(e.E for e in self._energies)

    @property
    def E_perp(self):
        return sum(e.E_perp for e in self._energies) * self.m_perp_factor

    @property
    def E_tot(self) -> float:
        return float(sum(e.E_tot for e in self._energies))

    def E_barrier(self, idx=None, min_only=False):
        """hotspice/core.py:625-656, evaluated on the device in FP64."""
        occ_inf = torch.as_tensor(self._occupation_inf, device=self.device)
        EB = torch.as_tensor(self._EB_np, device=self.device)
        dE = self.switch_energy() * occ_inf
        E = -dE / 2
        if not self.USE_PERP_ENERGY:
            if self.params.ENERGY_BARRIER_METHOD == 'simple':
                b = torch.maximum(dE, EB - E)
            else:
                b = torch.where(dE > 4 * EB, dE, torch.minimum(EB * (dE * (.25 / EB) + 1) ** 2, dE + 4 * EB))
            b1 = b2 = b
        else:
            Ep = self.perp_energy()
            b1 = torch.maximum(dE, EB + Ep - E)
            b2 = torch.maximum(dE, EB - Ep - E)
        if idx is not None:
            i = torch.as_tensor(np.asarray(idx), device=self.device, dtype=torch.long)
            b1, b2 = b1[i[0], i[1]], b2[i[0], i[1]]
        return torch.minimum(b1, b2) if min_only else (b1, b2)

    # observables ----------------------------------------------------------------------
    def _m_means(self) -> list:
        """Device scalars behind the magnetisation averages: the means of m ox and m oy for
        in-plane lattices, of m otherwise."""
        if self.in_plane:
            o = self._orient64()
            return [torch.mean(self.m * o[:, :, 0]), torch.mean(self.m * o[:, :, 1])]
        return [torch.mean(self.m)]

    def _m_avg_from(self, means) -> float:
        if not self.in_plane:
            return float(means[0])
        mx = float(means[0]) * self.nx * self.ny / self.n
        my = float(means[1]) * self.nx * self.ny / self.n
        return (mx ** 2 + my ** 2) ** 0.5

    @property
    def m_avg_x(self) -> float:
        if not self.in_plane:
            return 0
        return float(self._m_means()[0]) * self.nx * self.ny / self.n

    @property
    def m_avg_y(self) -> float:
        if not self.in_plane:
            return 0
        return float(self._m_means()[1]) * self.nx * self.ny / self.n

    @property
    def m_avg(self) -> float:
        return self._m_avg_from(self._m_means())

    def summary_async(self, keep_state: bool = False) -> 'RunSummary':
        """Enqueue on the current stream what a finished run's summary reads: the counters,
        the energy sums behind E_tot, the magnetisation means behind m_avg, the status words of
        enqueued recomputes, and the spins when ``keep_state``; all copied into pinned host
        memory. The host does not wait: RunSummary.ready() polls, result() gives the values
        (equal to the synchronous properties')."""
        torch_ = torch
        parts = [e.E_sum() for e in self._energies] + self._m_means()
        scal = torch_.stack([p.to(torch_.float64) for p in parts])
        pend, self._pending_status = getattr(self, '_pending_status', []), []
        host = {'scal': torch_.empty(scal.shape, dtype=torch_.float64, pin_memory=True),
                'counters': torch_.empty(self._counters.shape, dtype=self._counters.dtype, pin_memory=True)}
        host['scal'].copy_(scal, non_blocking=True)
        host['counters'].copy_(self._counters, non_blocking=True)
        if pend:
            st = torch_.stack([buf[n - 256:n - 252].view(torch_.int32)[0] for buf, n in pend])
            host['status'] = torch_.empty(st.shape, dtype=torch_.int32, pin_memory=True)
            host['status'].copy_(st, non_blocking=True)
        if keep_state:
            host['state'] = torch_.empty(self._m_dev.shape, dtype=self._m_dev.dtype, pin_memory=True)
            host['state'].copy_(self._m_dev, non_blocking=True)
        ev = torch_.cuda.Event()
        ev.record(torch_.cuda.current_stream(self.device))
        return RunSummary(self, host, [e.E_div for e in self._energies], ev)

    @property
    def m_avg_angle(self) -> float:
        return math.atan2(self.m_avg_y, self.m_avg_x) if self.in_plane else 0. + (self.m_avg < 0) * math.pi

    @property
    def T_avg(self) -> float:
        return float(np.mean(self._T_np))

    @property
    def E_B_avg(self) -> float:
        return float(np.mean(self._EB_np))

    @property
    def moment_avg(self) -> float:
        return float(np.mean(self._moment_np))

    def history_save(self, *, E_tot=None, t=None, T_avg=None, m_avg=None):
        self.history.entry(self)
        if E_tot is not None: self.history.E[-1] = float(E_tot)
        if t is not None: self.history.t[-1] = float(t)
        if T_avg is not None: self.history.T[-1] = float(T_avg)
        if m_avg is not None: self.history.m[-1] = float(m_avg)

    @lru_cache
    def calc_r(self, Q, as_scalar=True):
        """hotspice/core.py:720-733."""
        with np.errstate(divide='ignore'):
            r = (8e-7 * self._momentSq / (Q * self.kBT)) ** (1 / 3)
        r = np.clip(r, 0, (self.x_max - self.x_min) + (self.y_max - self.y_min))
        return float(np.max(r)) if as_scalar else r

    # ------------------------------------------------------------------ device plumbing
    def _dipolar(self):
        for e in self._energies:
            if isinstance(e, DipolarEnergy):
                return e
        return None

    def _lattice_struct(self, dip: DipolarEnergy | None = None):
        """HsLattice of the current state. ``dip`` overrides the registered dipolar energy
        (used while an energy is being initialised, before add_energy registers it)."""
        override = dip is not None and dip is not self._dipolar()
        if self._L is not None and not override:
            return self._L
        L = _lib.HsLattice()
        L.m = self._m_dev.data_ptr(); L.occ = self._occ_dev.data_ptr(); L.mm = self._mm_dev.data_ptr()
        L.moment = self._mom_dev.data_ptr(); L.nonzero = self._nonzero_dev.data_ptr()
        L.E_B = self._EB_dev.data_ptr(); L.beta = self._beta_dev.data_ptr()
        L.beta_uniform = self._beta_uniform
        L.m_perp_factor = self.m_perp_factor
        L.seed = self.seed
        L.nx, L.ny, L.ux, L.uy = self.nx, self.ny, self.unitcell.x, self.unitcell.y
        L.pbc = int(self.PBC); L.in_plane = int(self.in_plane); L.use_perp = int(self.USE_PERP_ENERGY)
        L.n_occ = self.n
        L.barrier_method = _lib.HS_BARRIER_SIMPLE if self.params.ENERGY_BARRIER_METHOD == 'simple' else _lib.HS_BARRIER_PARABOLIC
        L.trunc_cutoff = self.params.SIMULTANEOUS_SWITCHES_CONVOLUTION_OR_SUM_CUTOFF
        L.trunc_size = self.params.REDUCED_KERNEL_SIZE
        L.orient = _ptr(self._orient_dev)
        d = dip if override else self._dipolar()
        if d is not None:
            ks = d.kernel_set
            L.has_dipolar = 1
            L.K = d._K.data_ptr(); L.Kpo = _ptr(d._Kpo); L.Kps = _ptr(d._Kps)
            L.E_dip = d._E.data_ptr(); L.E_dip_perp = _ptr(d._Ep)
            L.sub_of = d._sub_of.data_ptr()
            L.dip_wx, L.dip_wy, L.dip_wrap, L.n_sub = ks.wx, ks.wy, int(ks.wrap), ks.K.shape[0]
            L.dip_pref = float(d.prefactor)
            L.dip_keep_perp_sign = int(d._keep_perp_sign)
        else:
            if not hasattr(self, '_sub_of_dummy'):
                self._sub_of_dummy = torch.full((self.unitcell.x * self.unitcell.y,), -1, device=self.device, dtype=torch.int32)
            L.sub_of = self._sub_of_dummy.data_ptr()
        for e in self._energies:
            if isinstance(e, ZeemanEnergy):
                L.zee = e._ef32.data_ptr()
                L.zee_perp = e._efp32.data_ptr()
            elif isinstance(e, ExchangeEnergy):
                nn = np.asarray(e.local_interaction, dtype=np.int64)
                L.has_exchange = 1
                L.J = float(e.J)
                L.nn_h, L.nn_w = nn.shape
                for i, v in enumerate(nn.reshape(-1)):
                    L.nn[i] = int(v)
                if self._beta_uniform > 0:
                    counts = np.arange(25, dtype=float)
                    kbt = np.full(25, kB * float(self._T_np[self.occupation.astype(bool)][0]))
                    bond = 1 - np.exp(-2 * e.J / kbt * counts)
                    self._bond_dev = to_device(bond, self.device, torch.float64)
                    L.wolff_bond = self._bond_dev.data_ptr()
        if not override:
            self._L = L
        return L

    def _switch_list(self, cap):
        sl = getattr(self, '_sw', None)
        if sl is None or sl[0].numel() < cap:
            cap = max(cap, 64)
            t = torch.zeros((3, cap), device=self.device, dtype=torch.int32)
            s = _lib.HsSwitchList()
            s.y, s.x, s.mode, s.cap = t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(), cap
            self._sw = (t, s)
            self._graphs.clear()
        return self._sw

    def _get_scratch(self, key, nbytes):
        buf = self._scratch.get(key)
        if buf is None or buf.numel() < nbytes:
            buf = torch.zeros(max(int(nbytes), 256), device=self.device, dtype=torch.uint8)
            self._scratch[key] = buf
            self._graphs.clear()
        return buf

    # -- full recompute and manual updates ----------------------------------------------
    def resync_energies(self, measure: bool = False):
        """Recompute the incrementally updated energies (the magnetostatic one) from the spins,
        with the configured full-recompute method (EngineConfig.recompute): the periodic resync
        that bounds the drift of the FP32 increments. Enqueued on the current stream; a status
        word of the tensor-core recompute is checked later (:meth:`check_resync`). With
        ``measure`` it returns the drift it removed, max |E_incremental - E_recomputed| /
        max |E_recomputed| (this synchronises); else None."""
        d = self._dipolar()
        if d is None:
            return 0.0 if measure else None
        before = d._E.clone() if measure else None
        self._full_recompute(d, check=False)
        if measure:
            return float((before - d._E).abs().max() / d._E.abs().max().clamp_min(1e-300))
        return None

    def check_resync(self):
        """Raise if a recompute enqueued by :meth:`resync_energies` reported a status
        (synchronises with it)."""
        pend, self._pending_status = getattr(self, '_pending_status', []), []
        for buf, nbytes in pend:
            st = int(buf[nbytes - 256:nbytes - 252].view(torch.int32).item())
            if st:
                raise RuntimeError(f'hs_dipolar_full_igemm reported status {st} (1: wait timed out, 2: moment not uniform)')

    def _full_recompute(self, d: DipolarEnergy, method=None, check=True):
        L = self._lattice_struct(d)
        method = method or self.engine.recompute
        ks = d.kernel_set
        N = self.nx * self.ny
        W = N if ks.full else (2 * ks.wx + 1) * (2 * ks.wy + 1)
        if method == 'auto':
            method = 'direct64' if N * W <= self.engine.direct_max_pairs or not self._igemm_ok(d) else 'igemm'
        elif method == 'igemm' and not self._igemm_ok(d):
            raise ValueError('igemm recompute needs the full uncropped kernel and a uniform moment')
        if method == 'direct64':
            _lib.check(self._lib.hs_dipolar_full_direct(L, 1, d._E.data_ptr(),
                                                        _ptr(d._Ep) if self.USE_PERP_ENERGY else None,
                                                        self._stream()), 'hs_dipolar_full_direct')
        elif method == 'direct32':
            _lib.check(self._lib.hs_dipolar_full_direct(L, 0, None, None, self._stream()), 'hs_dipolar_full_direct')
        elif method == 'igemm':
            nbytes = self._lib.hs_igemm_scratch_bytes(L, self.engine.igemm_splits)
            buf = self._get_scratch('igemm', max(nbytes, 1))
            _lib.check(self._lib.hs_dipolar_full_igemm(L, self.engine.igemm_splits, buf.data_ptr(), buf.numel(),
                                                        self._stream()), 'hs_dipolar_full_igemm')
            if not check:
                self._pending_status = getattr(self, '_pending_status', []) + [(buf, nbytes)]
                return
            st = int(buf[nbytes - 256:nbytes - 252].view(torch.int32).item())  # status word (synchronises)
            if st:
                raise RuntimeError(f'hs_dipolar_full_igemm reported status {st} (1: wait timed out, 2: moment not uniform)')
        else:
            raise ValueError(f"unknown recompute method '{method}'")

    def _igemm_ok(self, d) -> bool:
        """The implicit GEMM covers the full uncropped kernel and a uniform moment."""
        key = (self._version, id(d), id(d.kernel_set))
        hit = getattr(self, '_igemm_ok_cache', None)
        if hit is not None and hit[0] == key:
            return hit[1]
        ks = d.kernel_set
        ok = ks.wx == self.nx - 1 and ks.wy == self.ny - 1 and not ks.wrap
        if ok:
            mom = self._moment_np[self.occupation.astype(bool)]
            ok = mom.size == 0 or bool(np.all(mom == mom.flat[0]))
        self._igemm_ok_cache = (key, ok)
        return ok

    def _dipolar_apply(self, d, indices2D, semantics):
        idx = np.asarray(indices2D, dtype=np.int64).reshape(2, -1)
        k = idx.shape[1]
        if k == 0:
            return
        t, s = self._switch_list(k)
        t[0, :k].copy_(torch.as_tensor(idx[0], dtype=torch.int32))
        t[1, :k].copy_(torch.as_tensor(idx[1], dtype=torch.int32))
        if semantics == _lib.HS_UPDATE_MULTIPLE:
            ux, uy = self.unitcell.x, self.unitcell.y
            sub = (idx[1] % ux) + (idx[0] % uy) * ux
            counts = np.bincount(sub)
            mode = (counts[sub] > self.params.SIMULTANEOUS_SWITCHES_CONVOLUTION_OR_SUM_CUTOFF).astype(np.int32)
        else:
            mode = np.zeros(k, dtype=np.int32)
        t[2, :k].copy_(torch.as_tensor(mode))
        L = self._lattice_struct(d)
        _lib.check(self._lib.hs_dipolar_update(L, s, None, k, semantics, None, self._stream()), 'hs_dipolar_update')

    # ------------------------------------------------------------------ hot path
    def _grid_plan(self, r, scheme):
        key = (scheme, float(r))
        plan = self._plans.get(key)
        if plan is not None:
            return plan
        P = _lib.HsGridPlan()
        ux, uy = self.unitcell.x, self.unitcell.y
        tensors = []
        if scheme == 'grid':
            Rx = math.ceil(r / np.min(self.dx)) - 1
            Ry = math.ceil(r / np.min(self.dy)) - 1
            Rx, Ry = ux * math.ceil(Rx / ux), uy * math.ceil(Ry / uy)
            Rx, Ry = min(Rx, self.nx), min(Ry, self.ny)
            Rx, Ry = max(Rx, 2), max(Ry, 2)
            snx, sny = self.nx // Rx + 1, self.ny // Ry + 1
            n_sc = len(range(0, min(snx, self.nx), 2)) * len(range(0, min(sny, self.ny), 2))
            offs, packed = [0], []
            for ddy in range(uy):
                for ddx in range(ux):
                    oy, ox = self.occupation[ddy:ddy + Ry, ddx:ddx + Rx].nonzero()
                    packed.extend(((oy.astype(np.int64) << 16) | ox).tolist())
                    offs.append(len(packed))
            t_off = torch.as_tensor(np.asarray(offs, dtype=np.int32), device=self.device)
            t_yx = torch.as_tensor(np.asarray(packed if packed else [0], dtype=np.int32), device=self.device)
            tensors = [t_off, t_yx]
            P.phase_off, P.phase_yx = t_off.data_ptr(), t_yx.data_ptr()
            P.Rx, P.Ry, P.snx, P.sny, P.n_sc = Rx, Ry, snx, sny, n_sc
            P.sample_scheme = _lib.HS_SAMPLE_GRID
        elif scheme == 'single':
            P.sample_scheme = _lib.HS_SAMPLE_SINGLE
            P.n_sc = 1
        elif scheme == 'Poisson':
            P.sample_scheme = _lib.HS_SAMPLE_POISSON
            P.r_cells = float(r / min(np.min(self.dx), np.min(self.dy)))
            P.poisson_k = 4
            P.n_sc = 1
        else:
            raise ValueError(scheme)
        plan = (P, tensors)
        self._plans[key] = plan
        return plan

    def _step_args(self, kw):
        """Resolve the per-scheme launch arguments of one update step."""
        sch = self.params.UPDATE_SCHEME
        L = self._lattice_struct()
        if sch == Scheme.NEEL:
            af = float(kw.get('attempt_freq', 1e10))
            nbytes = self._lib.hs_neel_scratch_bytes(L)
            buf = self._get_scratch('neel', nbytes)
            t, s = self._switch_list(1)
            return ('neel', L, s, af, buf)
        if sch == Scheme.METROPOLIS:
            if kw.get('idx') is not None:
                raise NotImplementedError('_update_Metropolis(idx=...) with caller-chosen indices is not on the device path')
            ms = self.params.MULTISAMPLING_SCHEME
            if ms == 'cluster':
                raise ValueError("MULTISAMPLING_SCHEME='cluster' needs UPDATE_SCHEME=Wolff")
            Q = kw.get('Q', 0.05)
            r = kw.get('r', 0)
            r = self.calc_r(Q) if r == 0 else r
            P, _ = self._grid_plan(r, ms)
            P.metropolis_time = int(self.params.METROPOLIS_TIME)
            P.attempt_freq = float(kw.get('attempt_freq', 1e10))
            nbytes = self._lib.hs_metropolis_scratch_bytes(L, P)
            buf = self._get_scratch(('metro', ms, float(r)), nbytes)
            cap = max(P.n_sc, 1)
            if ms == 'Poisson':
                cap = max(cap, (nbytes // 20) + 1)
            t, s = self._switch_list(cap)
            return ('metro', L, s, P, buf)
        if sch == Scheme.WOLFF:
            nbytes = self._lib.hs_wolff_scratch_bytes(L)
            buf = self._get_scratch('wolff', nbytes)
            t, s = self._switch_list(self.nx * self.ny)
            return ('wolff', L, s, None, buf)
        raise ValueError(f"The Magnets.params object has an invalid value for UPDATE_SCHEME='{sch}'.")

    def _launch(self, args, stream):
        kind, L, s, extra, buf = args
        C = self._counters.data_ptr()
        if kind == 'neel':
            rc = self._lib.hs_neel_step(L, C, s, extra, buf.data_ptr(), buf.numel(), stream)
        elif kind == 'metro':
            rc = self._lib.hs_metropolis_step(L, C, s, extra, buf.data_ptr(), buf.numel(), stream)
        else:
            rc = self._lib.hs_wolff_step(L, C, s, buf.data_ptr(), buf.numel(), stream)
        _lib.check(rc, f'hs_{kind}_step')

    def update(self, *args, **kwargs):
        """One update step (hotspice/core.py:604-622). Returns the switched index/indices."""
        if self._T_zero:
            if self.params.UPDATE_SCHEME != Scheme.METROPOLIS:
                warnings.warn("T=0 somewhere in the domain, so no switch will be simulated to prevent DIV/0 errors.", stacklevel=2)
            else:
                warnings.warn("T=0 somewhere in the domain, so ergodicity can not be guaranteed. Proceed with caution.", stacklevel=2)
            return None
        if self.params.UPDATE_SCHEME == Scheme.NEEL:
            self._write_counters(t_max=float(kwargs.get('t_max', 1)), progress=0, done=0)
        args_ = self._step_args(kwargs)
        self._launch(args_, self._stream())
        c = self._read_counters()
        n = int(c['n_sw'])
        t, _ = self._sw
        if self.params.UPDATE_SCHEME == Scheme.NEEL:
            if n == 0:
                return None
            yx = t[:2, 0].cpu().numpy()
            return (int(yx[0]), int(yx[1]))
        idx = t[:2, :n].cpu().numpy().astype(np.int64)
        if self.params.UPDATE_SCHEME == Scheme.WOLFF:
            order = np.lexsort((idx[1], idx[0]))
            idx = idx[:, order]
        return idx

    def progress(self, t_max: float = 1, MCsteps_max: float = 4., stepwise: bool = False, **kwargs):
        """hotspice/core.py:736-760. Non-stepwise runs execute on the device in chunks of
        ``EngineConfig.graph_steps`` steps (CUDA-graph replays) and synchronise per chunk."""
        check_progress_limits(t_max, MCsteps_max)
        if stepwise:
            return self._progress_stepwise(t_max=t_max, MCsteps_max=MCsteps_max, **kwargs)
        if self._T_zero:
            raise RuntimeError('progress() with T=0 somewhere in the domain would never advance')
        if self.engine.persistent:
            from .engine import BatchEngine
            return BatchEngine([self], cluster_size=self.engine.cluster_size or None).progress(
                t_max=t_max, MCsteps_max=MCsteps_max, **kwargs)[0]
        c = self._read_counters()
        t0 = float(c['t'])
        mc0 = float(c['attempted']) / self.n
        self._write_counters(t0=t0, mc0=mc0, t_max=float(t_max), mc_max=float(MCsteps_max), progress=1, done=0)
        self._run_until_done(kwargs)
        c = self._read_counters()
        self._write_counters(progress=0, done=0)
        return float(c['t']) - t0, float(c['attempted']) / self.n - mc0

    def _run_until_done(self, kw, max_chunks=10 ** 9):
        args_ = self._step_args(kw)
        K = max(1, int(self.engine.graph_steps))
        off_done = _lib.HsCounters.done.offset
        steps_since_resync = 0
        for _ in range(max_chunks):
            self._run_chunk(args_, K)
            steps_since_resync += K
            if self.engine.resync_every and steps_since_resync >= self.engine.resync_every:
                d = self._dipolar()
                if d is not None:
                    self._full_recompute(d)
                steps_since_resync = 0
            flag = int(self._counters[off_done:off_done + 4].cpu().view(torch.int32)[0])
            if flag:
                break
            st = int(self._counters[_lib.HsCounters.status.offset:_lib.HsCounters.status.offset + 4].cpu().view(torch.int32)[0])
            if st:
                raise RuntimeError(f'device step reported status {st} (HS_ST_* bits)')

    def _run_chunk(self, args_, K):
        if not self.engine.use_graphs:
            st = self._stream()
            for _ in range(K):
                self._launch(args_, st)
            return
        extra = args_[3]
        extra_key = extra if isinstance(extra, float) or extra is None else (extra.sample_scheme, extra.Rx, extra.Ry,
                                                                            extra.r_cells, extra.metropolis_time,
                                                                            extra.attempt_freq, extra.phase_yx)
        key = (args_[0], extra_key, args_[4].data_ptr(), self._sw[0].data_ptr(), self._version, K)
        g = self._graphs.get(key)
        if g is None:
            # warm-up launch outside capture is not needed: every launch is a plain kernel
            g = torch.cuda.CUDAGraph()
            s = torch.cuda.Stream(self.device)
            s.wait_stream(torch.cuda.current_stream(self.device))
            with torch.cuda.graph(g, stream=s):
                for _ in range(K):
                    self._launch(args_, s.cuda_stream)
            torch.cuda.current_stream(self.device).wait_stream(s)
            self._graphs[key] = g
        g.replay()

    def run(self, steps: int, **kwargs):
        """Engine extension (no reference counterpart): enqueue exactly ``steps`` update steps
        of the current scheme on the device, without the progress() stop rule and without any
        host synchronisation. Returns immediately; read counters / state to synchronise."""
        if self._T_zero:
            raise RuntimeError('run() with T=0 somewhere in the domain')
        if self.engine.persistent:
            self._engine_run(int(steps), kwargs)
            return
        self._set_control(progress=0, done=0, t_max=float(kwargs.pop('t_max', math.inf)))
        args_ = self._step_args(kwargs)
        K = max(1, int(self.engine.graph_steps))
        q, r = divmod(int(steps), K)
        for _ in range(q):
            self._run_chunk(args_, K)
        if r:
            self._run_chunk(args_, r)

    def _engine_run(self, steps, kwargs):
        from .engine import BatchEngine
        kw = dict(kwargs)
        t_max = float(kw.pop('t_max', math.inf))
        key = (steps, tuple(sorted((k, float(v)) for k, v in kw.items())), self._version, t_max,
               self.engine.cluster_size)
        cache = getattr(self, '_engine_cache', None)
        if cache is None or cache[0] != key:
            eng = BatchEngine([self], cluster_size=self.engine.cluster_size or None)
            self._set_control(progress=0, done=0, t_max=t_max)
            prepared = eng._prepare([steps], [kw])
            self._engine_cache = cache = (key, eng, prepared)
        else:
            self._set_control(progress=0, done=0, t_max=t_max)
        cache[1].launch(cache[2])

    # ------------------------------------------------------------------ device-side stepping
    def _moment64(self):
        """FP64 device copy of the moment (the Zeeman factors are formed from it on the device)."""
        c = getattr(self, '_mom64_cache', None)
        if c is None or c[0] is not self._moment_np:
            c = (self._moment_np, to_device(self._moment_np, self.device, torch.float64))
            self._mom64_cache = c
        return c[1]

    def _orient64(self):
        c = getattr(self, '_ori64_cache', None)
        if c is None or c[0] is not self.orientation:
            c = (self.orientation, to_device(self.orientation, self.device, torch.float64))
            self._ori64_cache = c
        return c[1]

    def _progress_enqueue(self, t_max: float = 1, MCsteps_max: float = 4., **kwargs):
        """progress(t_max, MCsteps_max) enqueued on the current stream with no host round trip:
        hs_progress_arm sets the stop rule from the device counters, then one persistent engine
        launch steps until it holds. Call :meth:`_progress_finish` after the last one (it ends
        the armed state). Without the persistent engine this falls back to progress()."""
        check_progress_limits(t_max, MCsteps_max)
        if not self.engine.persistent:
            self.progress(t_max=t_max, MCsteps_max=MCsteps_max, **kwargs)
            return
        if self._T_zero:
            raise RuntimeError('progress() with T=0 somewhere in the domain would never advance')
        from .engine import BatchEngine
        key = (self._version, tuple(sorted((k, float(v)) for k, v in kwargs.items())), self.engine.cluster_size)
        c = getattr(self, '_pe_cache', None)
        if c is None or c[0] != key:
            eng = BatchEngine([self], cluster_size=self.engine.cluster_size or None)
            c = (key, eng, eng._prepare([0], [dict(kwargs)]))
            self._pe_cache = c
        self._progress_arm(t_max, MCsteps_max)
        c[1].launch(c[2])

    def _progress_arm(self, t_max: float, MCsteps_max: float):
        """Arm progress(t_max, MCsteps_max) on the device (hs_progress_arm); the next engine
        launch that runs this instance steps until the stop rule holds."""
        _lib.check(self._lib.hs_progress_arm(self._counters.data_ptr(), self.n, float(t_max), float(MCsteps_max),
                                             self._stream()), 'hs_progress_arm')
        self._ctl = None      # the device wrote t_max / progress / done: the host-side cache is stale

    def _progress_finish(self):
        """End device-armed progress() runs: plain steps run again; raises on a device status."""
        _lib.check(self._lib.hs_progress_disarm(self._counters.data_ptr(), self._stream()), 'hs_progress_disarm')
        self._ctl = None
        st = int(self._read_counters()['status'])
        if st:
            raise RuntimeError(f'device step reported status {st} (HS_ST_* bits)')

    # ------------------------------------------------------------------ relaxation
    def _relax_args(self):
        L = self._lattice_struct()
        nbytes = self._lib.hs_relax_scratch_bytes(L)
        if nbytes < 0:
            _lib.check(-1, 'hs_relax_scratch_bytes')
        buf = self._get_scratch('relax', nbytes)
        _, s = self._switch_list(self.nx * self.ny)
        return L, s, buf

    @staticmethod
    def _relax_word(buf, k):
        """Word k of the relax scratch's header: 0 = stop rule fired, 1 = sweeps made."""
        return int(buf[4 * k:4 * k + 4].cpu().view(torch.int32)[0])

    def _replay(self, key, enqueue):
        """Run ``enqueue(stream)`` once, as a CUDA graph when graphs are enabled (cached under
        ``key``; every kernel it launches reads its control state from device memory)."""
        if not self.engine.use_graphs:
            enqueue(self._stream())
            return
        g = self._graphs.get(key)
        if g is None:
            g = torch.cuda.CUDAGraph()
            s = torch.cuda.Stream(self.device)
            s.wait_stream(torch.cuda.current_stream(self.device))
            with torch.cuda.graph(g, stream=s):
                enqueue(s.cuda_stream)
            torch.cuda.current_stream(self.device).wait_stream(s)
            self._graphs[key] = g
        g.replay()

    def _minimize_all(self, ignore_barrier=True, _simultaneous=False):
        """hotspice/core.py:799-825: one sweep over the (2 ux) x (2 uy) subgrids in a random
        order (one Philox call), switching in each subgrid every magnet whose switch lowers
        the energy (or, without ignore_barrier, whose switch_energy/2 + E_B < 0)."""
        if _simultaneous:
            warnings.warn("_simultaneous=True in _minimize_all(). I hope you know what you are doing, as this is very nonphysical ;)", stacklevel=2)
        L, s, buf = self._relax_args()
        st = self._stream()
        _lib.check(self._lib.hs_relax_begin(L, buf.data_ptr(), buf.numel(), st), 'hs_relax_begin')
        _lib.check(self._lib.hs_minimize_all(L, self._counters.data_ptr(), s, int(bool(ignore_barrier)),
                                             int(bool(_simultaneous)), buf.data_ptr(), buf.numel(), st),
                   'hs_minimize_all')

    def relax(self, verbose=False, **kwargs):
        """hotspice/core.py:827-861: _minimize_all sweeps until one switches nothing, the state
        equals the one two sweeps before, or int(sqrt(nx^2 + ny^2)) sweeps were made. The
        sweeps and the stop rule run on the device (``EngineConfig.graph_steps`` sweeps per
        CUDA-graph replay, one host check per replay). Returns nothing, like the reference;
        the number of sweeps is kept in ``self.relax_sweeps``."""
        ignore_barrier = bool(kwargs.pop('ignore_barrier', True))
        simultaneous = bool(kwargs.pop('_simultaneous', False))
        if kwargs:
            raise TypeError(f"relax() got unexpected keyword arguments {sorted(kwargs)}")
        if simultaneous:
            warnings.warn("_simultaneous=True in _minimize_all(). I hope you know what you are doing, as this is very nonphysical ;)", stacklevel=2)
        n_max = int(math.sqrt(self.nx ** 2 + self.ny ** 2))
        self.relax_sweeps = 0
        if not bool(torch.any(self._m_dev != 0)):   # allclose(zeros, m): the loop never starts
            return
        L, s, buf = self._relax_args()
        lib, C = self._lib, self._counters.data_ptr()
        st = self._stream()
        _lib.check(lib.hs_relax_begin(L, buf.data_ptr(), buf.numel(), st), 'hs_relax_begin')
        P = 1 if simultaneous else 4 * self.unitcell.x * self.unitcell.y
        K = max(1, min(int(self.engine.graph_steps), n_max, 2048 // (3 * P + 3)))   # about 2k graph nodes

        def sweeps(stream):
            for _ in range(K):
                _lib.check(lib.hs_minimize_all(L, C, s, int(ignore_barrier), int(simultaneous), buf.data_ptr(),
                                               buf.numel(), stream), 'hs_minimize_all')
                _lib.check(lib.hs_relax_check(L, C, n_max, buf.data_ptr(), buf.numel(), stream), 'hs_relax_check')
        key = ('relax', ignore_barrier, simultaneous, K, buf.data_ptr(), s.y, self._version)
        for _ in range((n_max + K - 1) // K):
            self._replay(key, sweeps)
            if self._relax_word(buf, 0):
                break
        self.relax_sweeps = self._relax_word(buf, 1)
        if verbose:
            print(f"Used {self.relax_sweeps} (out of {n_max}) steps in relax().")

    def minimize(self, ignore_barrier=True, verbose=False, _frac=0.3):
        """hotspice/core.py:763-797, on the device: per iteration, with n magnets gaining more
        than kBT by switching, ceil(frac n) of them switch (one Philox call chooses them);
        otherwise the magnet with the most to gain switches, unless nothing gains or it was
        picked a third time. ``ignore_barrier=False`` is refused: there the reference compares
        the (barrier, barrier) tuple returned by E_barrier() and indexes the result as if it
        were one array."""
        if not ignore_barrier:
            raise NotImplementedError('minimize(ignore_barrier=False) has no well-defined reference result')
        L, s, buf = self._relax_args()
        lib, C = self._lib, self._counters.data_ptr()
        st = self._stream()
        _lib.check(lib.hs_minimize_begin(L, buf.data_ptr(), buf.numel(), st), 'hs_minimize_begin')
        K = max(1, int(self.engine.graph_steps))
        frac = float(_frac)

        def iterations(stream):
            for _ in range(K):
                _lib.check(lib.hs_minimize_step(L, C, s, frac, buf.data_ptr(), buf.numel(), stream), 'hs_minimize_step')
        key = ('minimize', frac, K, buf.data_ptr(), s.y, self._version)
        while True:
            self._replay(key, iterations)
            if self._relax_word(buf, 0):
                break

    def _snapshot(self):
        d = self._dipolar()
        return {'m': self._m_dev.clone(), 'mm': self._mm_dev.clone(), 'C': self._counters.clone(),
                'E': d._E.clone() if d is not None else None,
                'Ep': d._Ep.clone() if d is not None and d._Ep is not None else None}

    def _restore(self, snap):
        d = self._dipolar()
        self._m_dev.copy_(snap['m']); self._mm_dev.copy_(snap['mm']); self._counters.copy_(snap['C'])
        if d is not None:
            d._E.copy_(snap['E'])
            if snap['Ep'] is not None:
                d._Ep.copy_(snap['Ep'])
        self._ctl = None

    def _progress_stepwise(self, t_max: float = 1, MCsteps_max: float = 4., **kwargs):
        t_0, MCsteps_0 = self.t, self.MCsteps
        while lower_than(dt := self.t - t_0, t_max) and lower_than(self.MCsteps - MCsteps_0, MCsteps_max):
            if self.params.UPDATE_SCHEME == Scheme.NEEL:
                self.update(t_max=(t_max - dt), **kwargs)
            else:
                self.update(**kwargs)
            yield
        return self.t - t_0, self.MCsteps - MCsteps_0

    # ------------------------------------------------------------------ subclass hooks
    def _get_angles(self):
        return np.zeros_like(self.ixx, dtype=float)

    def _get_occupation(self):
        return np.ones_like(self.ixx)

    def _get_groundstate(self):
        return 'random'

    def _get_nearest_neighbors(self):
        return np.array([[0, 1, 0], [1, 0, 1], [0, 1, 0]])

    def _get_appropriate_avg(self):
        return 'cross'

    def _get_AFMmask(self):
        return np.array([[1, 0, -1], [0, 0, 0], [-1, 0, 1]], dtype='float')
