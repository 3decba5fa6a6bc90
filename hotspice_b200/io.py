"""Reservoir-computing inputs and outputs with the interface of hotspice/io.py:20-500, stepping
on the device.

An input (``Inputter.input_single``) sets the Zeeman field and runs progress() or minimize();
an output (``OutputReader.read_state``) coarse-grains the spins. Here the field is written in
place on the device (``ZeemanEnergy.set_field_device`` -> hs_zeeman_set), progress() is armed
on the device and run by one persistent engine launch until its stop rule holds
(``Magnets._progress_enqueue`` -> hs_progress_arm + hs_engine_run), and the regional readouts
are one CTA per region (hs_region_readout). :func:`run_sequence` drives a whole input sequence
that way and synchronises once, at the end. Inputs that need the host between steps (the
sinusoidal FieldInputter, PerpFieldInputter with relax=True, which runs minimize()) use the
same device operations from a host loop.

Datastreams draw on the host (numpy Generators, as the reference does with ``xp.random``); the
values only choose launch parameters. State arrays come back as float64 torch tensors on the
simulation's device.
"""
from __future__ import annotations

import math
import warnings
from abc import ABC, abstractmethod
from inspect import isgeneratorfunction
from typing import Literal

import numpy as np
import torch

from . import _lib
from .ASI import OOP_Square
from .core import Magnets, Scheme
from .energies import ZeemanEnergy
from .utils import lower_than

__all__ = ['Datastream', 'ScalarDatastream', 'BinaryDatastream', 'IntegerDatastream', 'ConstantDatastream',
           'RandomBinaryDatastream', 'RandomIntegerDatastream', 'RandomScalarDatastream', 'Inputter', 'OutputReader',
           'FieldInputter', 'FieldInputterBinary', 'PerpFieldInputter', 'FullOutputReader', 'RegionalOutputReader',
           'OOPSquareChessFieldInputter', 'OOPSquareChessOutputReader', 'OOPSquareChessStepsInputter', 'Stage',
           'run_sequence', 'run_batch']


# ------------------------------------------------------------------------------ datastreams
class Datastream(ABC):
    """hotspice/io.py:20-35."""

    def __init__(self):
        self.rng = np.random.default_rng(None)

    def reset_rng(self):
        self.rng = np.random.default_rng(0)

    @abstractmethod
    def get_next(self, n=1) -> np.ndarray:
        """Exactly ``n`` scalar values."""

    @property
    @abstractmethod
    def dtype(self):
        return None


class ScalarDatastream(Datastream):
    @property
    def dtype(self):
        return float


class BinaryDatastream(Datastream):
    @property
    def dtype(self):
        return int


class IntegerDatastream(Datastream):
    @property
    def dtype(self):
        return int

    @property
    @abstractmethod
    def bits_per_int(self) -> int:
        pass

    def as_bits(self, integer: int, endianness: Literal['little', 'big'] = 'little') -> np.ndarray:
        """hotspice/io.py:55-61: the binary digits, least significant first by default."""
        bits = bin(integer)[2:].zfill(self.bits_per_int)
        if endianness == 'little':
            bits = bits[::-1]
        return np.asarray([int(b) for b in bits])


class ConstantDatastream(ScalarDatastream):
    def __init__(self, constant: float = 1):
        super().__init__()
        self.constant = constant

    def get_next(self, n=1) -> np.ndarray:
        return np.ones(n, dtype=float) * self.constant

    def __repr__(self):
        return f"hotspice.io.ConstantDatastream(constant={self.constant})"


class RandomBinaryDatastream(BinaryDatastream):
    """hotspice/io.py:144-155: 0 with probability p0, else 1."""

    def __init__(self, p0=.5):
        self.p0 = p0
        super().__init__()

    def __repr__(self):
        return f"hotspice.io.RandomBinaryDatastream(p0={self.p0})"

    def get_next(self, n=1) -> np.ndarray:
        return self.rng.random(size=(n,)) >= self.p0


class RandomIntegerDatastream(IntegerDatastream):
    """hotspice/io.py:157-179: uniform integers in [0, 2**num_bits)."""

    def __init__(self, num_bits: int = 8):
        if not isinstance(num_bits, int):
            raise ValueError("Number of bits per 'byte' in RandomUniformByteDatastream must be of type <int>.")
        self.num_bits = num_bits
        self._max = 2 ** self.num_bits
        super().__init__()

    def __repr__(self):
        return f"hotspice.io.RandomIntegerDatastream(num_bits={self.num_bits})"

    @property
    def bits_per_int(self) -> int:
        return self.num_bits

    def get_next(self, n=1) -> np.ndarray:
        return self.rng.integers(0, self._max, size=(n,))


class RandomScalarDatastream(ScalarDatastream):
    def __init__(self, low=0, high=1):
        self.low, self.high = low, high
        super().__init__()

    def __repr__(self):
        return f"hotspice.io.RandomScalarDatastream(low={self.low}, high={self.high})"

    def get_next(self, n=1) -> np.ndarray:
        return (self.high - self.low) * self.rng.random(size=(n,)) + self.low


# ------------------------------------------------------------------------------ base classes
def _zeeman(mm: Magnets) -> ZeemanEnergy:
    Zeeman = mm.get_energy('Zeeman')
    if Zeeman is None:
        mm.add_energy(Zeeman := ZeemanEnergy(0, 0))
    return Zeeman


def _expand(inputter, values):
    """The values input_single receives: integers of an IntegerDatastream become their bits."""
    if isinstance(inputter.datastream, IntegerDatastream):
        return np.asarray([inputter.datastream.as_bits(int(v)) for v in values]).reshape(-1)
    return values


class Stage:
    """One field-then-progress step of an input: the Zeeman field magnitude * pattern (pattern
    None: uniform) at ``angle`` (None: unchanged), then progress(t_max, MCsteps_max)."""
    __slots__ = ('magnitude', 'pattern', 'angle', 't_max', 'mc_max')

    def __init__(self, magnitude, pattern, angle, t_max, mc_max):
        self.magnitude, self.pattern, self.angle, self.t_max, self.mc_max = magnitude, pattern, angle, t_max, mc_max


def _run_stages(mm: Magnets, stages):
    Zeeman = _zeeman(mm)
    for st in stages:
        Zeeman.set_field_device(st.magnitude, pattern=st.pattern, angle=st.angle)
        mm._progress_enqueue(t_max=st.t_max, MCsteps_max=st.mc_max)


class Inputter(ABC):
    """hotspice/io.py:73-106."""

    def stages(self, mm: Magnets, value):
        """The input of ``value`` as a list of :class:`Stage`, or None when it needs the host
        between steps (then only input_single applies it)."""
        return None

    def __init__(self, datastream: Datastream = None):
        self.datastream = ConstantDatastream(constant=1) if datastream is None else datastream

    def input(self, mm: Magnets, values=None, remove_stimulus=False) -> np.ndarray:
        if values is None:
            values = self.datastream.get_next(n=1)
        values = np.asarray(values).reshape(-1)
        gen = isgeneratorfunction(self.input_single)
        for value in _expand(self, values.copy()):
            result = self.input_single(mm, value)
            if gen:
                for _ in result:
                    pass
        if remove_stimulus:
            self.remove_stimulus(mm)
        mm._progress_finish()
        return values

    def remove_stimulus(self, mm: Magnets):
        mm.get_energy('Zeeman').set_field_device(0.0)

    @abstractmethod
    def input_single(self, mm: Magnets, value: float | int | bool):
        """Applies the stimulus for one scalar value (a function or a generator)."""


class OutputReader(ABC):
    """hotspice/io.py:109-138."""

    def __init__(self, mm: Magnets = None):
        self.mm = mm
        if mm is not None:
            self.configure_for(mm)

    def configure_for(self, mm: Magnets):
        self.mm = mm

    @abstractmethod
    def read_state(self, mm: Magnets = None) -> torch.Tensor:
        if (mm is not None) and (mm is not self.mm):
            self.configure_for(mm)

    def read_into(self, mm: Magnets, out: torch.Tensor):
        """Write the readout of ``mm``'s current state into the device tensor ``out`` (n values),
        asynchronously."""
        out.copy_(self.read_state(mm))

    @property
    def n(self) -> int:
        return int(self.state.numel())

    @property
    def node_coords(self) -> np.ndarray:
        return self._node_coords


# ------------------------------------------------------------------------------ inputters
class FieldInputter(Inputter):
    """hotspice/io.py:193-239: a field of magnitude * value at ``angle``, for at most ``n``
    Monte Carlo steps per input (half a period, or a full +/- period)."""

    def __init__(self, datastream: Datastream, magnitude=1, angle=0, n=2, sine=False, frequency=1, half_period=True):
        super().__init__(datastream)
        self.angle = angle
        self.magnitude = magnitude
        self.n = n
        self.sine = sine
        self.frequency = frequency
        self.half_period = half_period

    @property
    def angle(self):
        return self._angle

    @angle.setter
    def angle(self, value):
        self._angle = value % math.tau

    @property
    def full_period(self):
        return not self.half_period

    def stages(self, mm: Magnets, value):
        if self.sine:
            return None
        angle = self.angle if mm.in_plane else None
        period = 1 / (1 + self.half_period)
        out = [Stage(self.magnitude * value, None, angle, 1 / self.frequency / (2 * period), self.n / (2 * period))]
        if self.full_period:
            out.append(Stage(-self.magnitude * value, None, None, .5 / self.frequency, self.n / 2))
        return out

    def input_single(self, mm: Magnets, value: float | int):
        if self.sine and mm.params.UPDATE_SCHEME != Scheme.NEEL:
            raise AttributeError("Can not use temporal sine=True if UPDATE_SCHEME != Scheme.NEEL.")
        Zeeman = _zeeman(mm)
        angle = self.angle if mm.in_plane else None
        period = 1 / (1 + self.half_period)
        if self.sine:
            # the field follows the sine step by step: a host loop over device steps
            mm._progress_finish()
            Zeeman.set_field(angle=angle)
            MCsteps0, t0 = mm.MCsteps, mm.t
            while lower_than(progress := max((mm.MCsteps - MCsteps0) / self.n, (mm.t - t0) * self.frequency), 1):
                Zeeman.set_field_device(self.magnitude * value * math.sin(progress * math.pi * 2 * period))
                mm.update(t_max=min(1 - progress, 0.05) / self.frequency)
        else:
            _run_stages(mm, self.stages(mm, value))


class FieldInputterBinary(FieldInputter):
    """hotspice/io.py:242-256: magnitude magnitudes[1] for a 1, magnitudes[0] for a 0."""

    def __init__(self, datastream: Datastream, magnitudes: tuple = (.8, 1), **kwargs):
        self.magnitude_ratio = magnitudes[0] / magnitudes[1]
        super().__init__(datastream, magnitude=magnitudes[1], half_period=False, **kwargs)

    def stages(self, mm: Magnets, value):
        return super().stages(mm, 1 if value else self.magnitude_ratio)

    def input_single(self, mm: Magnets, value: bool | int):
        super().input_single(mm, 1 if value else self.magnitude_ratio)


class PerpFieldInputter(FieldInputter):
    """hotspice/io.py:259-309: the bit chooses the field angle (angle or angle + pi/2); a +/-
    field pair, each followed by minimize() (relax=True) or by progress()."""

    def __init__(self, datastream: BinaryDatastream, magnitude=1, angle=0, n=2, relax=True, frequency=1, **kwargs):
        self.relax = relax
        super().__init__(datastream, magnitude=magnitude, angle=angle, n=n, frequency=frequency)

    def _check(self, mm):
        if (self.sine or self.frequency) and mm.params.UPDATE_SCHEME != Scheme.NEEL:
            raise AttributeError("Can not use temporal sine=True or nonzero frequency if UPDATE_SCHEME != Scheme.NEEL.")
        if not mm.in_plane:
            raise AttributeError("Can not use PerpFieldInputter on an out-of-plane ASI.")

    def stages(self, mm: Magnets, value):
        if self.relax:
            return None
        self._check(mm)
        angle = self.angle + value * math.pi / 2
        return [Stage(self.magnitude, None, angle, 0.5 / self.frequency, self.n),
                Stage(-self.magnitude, None, angle, 0.5 / self.frequency, self.n)]

    def input_single(self, mm: Magnets, value: bool | int):
        self._check(mm)
        if self.relax:
            Zeeman = _zeeman(mm)
            angle = self.angle + value * math.pi / 2
            for mag in [self.magnitude, -self.magnitude]:
                Zeeman.set_field_device(mag, angle=angle)
                mm.minimize()
        else:
            _run_stages(mm, self.stages(mm, value))

    def input_single_generalized(self, mm: Magnets, value: bool | int):
        self._check(mm)
        Zeeman = _zeeman(mm)
        angle = self.angle + value * math.pi / 2
        if self.sine:
            mm._progress_finish()
            MCsteps0, t0 = mm.MCsteps, mm.t
            while lower_than(progress := max((mm.MCsteps - MCsteps0) / self.n, (mm.t - t0) * self.frequency), 1):
                Zeeman.set_field_device(self.magnitude * math.sin(progress * math.pi * (2 - self.half_period)), angle=angle)
                mm.update(t_max=min(1 - progress, 0.125) / self.frequency)
        else:
            Zeeman.set_field_device(self.magnitude, angle=angle)
            mm._progress_enqueue(t_max=1 / self.frequency, MCsteps_max=self.n)


def _checkerboard(mm: Magnets, kind: str) -> torch.Tensor:
    """k = (ixx + iyy) % 2 as an FP32 device pattern: 'pm' 2k - 1, '01' k, 'm10' k - 1."""
    key = '_chess_' + kind
    t = getattr(mm, key, None)
    if t is None:
        a = ((mm.ixx + mm.iyy) % 2).astype(float)
        a = {'pm': a * 2 - 1, '01': a, 'm10': a - 1}[kind]
        t = torch.as_tensor(a, device=mm.device, dtype=torch.float32).contiguous()
        setattr(mm, key, t)
    return t


class OOPSquareChessFieldInputter(Inputter):
    """hotspice/io.py:382-401: a checkerboard field AFM_mask * (2 value - 1) * magnitude."""

    def __init__(self, datastream: Datastream, magnitude: float = 1, n=4, frequency=1):
        super().__init__(datastream)
        self.magnitude = magnitude
        self.n = n
        self.frequency = frequency

    def stages(self, mm: OOP_Square, value):
        return [Stage((2 * value - 1) * self.magnitude, _checkerboard(mm, 'pm'), None, 1 / self.frequency, self.n)]

    def input_single(self, mm: OOP_Square, value: bool | int):
        _run_stages(mm, self.stages(mm, value))


class OOPSquareChessStepsInputter(Inputter):
    """hotspice/io.py:448-500: the two halves of the checkerboard, one after the other, with a
    magnitude that is a piecewise-linear function of a scalar value (or +/- magnitude for bits)."""

    def __init__(self, datastream: Datastream, magnitude: float = 1., magnitude_range: float = 0.,
                 transition_range: float = 1., n: float = 4., frequency: float = 1.):
        super().__init__(datastream)
        self.magnitude, self.magnitude_range, self.transition_range = magnitude, magnitude_range, transition_range
        self.n = n
        self.frequency = frequency
        self.transform = self._get_transform_func()

    def stages(self, mm: OOP_Square, value):
        magnitude = self.transform(value)
        return [Stage(magnitude, _checkerboard(mm, '01'), None, 1 / self.frequency, self.n),     # 0 / 1 checkerboard
                Stage(magnitude, _checkerboard(mm, 'm10'), None, 1 / self.frequency, self.n)]   # -1 / 0, the other half

    def input_single(self, mm: OOP_Square, value: float | int | bool):
        _run_stages(mm, self.stages(mm, value))

    def _get_transform_func(self):
        if isinstance(self.datastream, (BinaryDatastream, IntegerDatastream)):
            return lambda bit: (2 * bit - 1) * self.magnitude
        if isinstance(self.datastream, ScalarDatastream):
            return self._val_to_mag_piecewiselinear

    def _val_to_mag_piecewiselinear(self, value: float):
        s = 0.5 - self.transition_range / 2
        if value < s:
            return -self.magnitude + value * self.magnitude_range / s
        if value > 1 - s:
            return self.magnitude + (value - 1) * self.magnitude_range / s
        return 2 * (self.magnitude - self.magnitude_range) / self.transition_range * (value - 0.5)


# ------------------------------------------------------------------------------ readers
class FullOutputReader(OutputReader):
    """hotspice/io.py:312-332: the spins of the occupied cells."""

    def configure_for(self, mm: Magnets):
        self.mm = mm
        self.indices = mm.nonzero
        self._flat = torch.as_tensor(np.ravel_multi_index(self.indices, (mm.ny, mm.nx)), device=mm.device, dtype=torch.long)
        self.state = mm._m_dev.reshape(-1)[self._flat].double()
        self._node_coords = np.asarray([mm.xx[self.indices], mm.yy[self.indices]]).T

    def read_state(self, mm: Magnets = None, m=None) -> torch.Tensor:
        super().read_state(mm)
        if m is None:
            self.state = self.mm._m_dev.reshape(-1)[self._flat].double()
        else:
            self.state = torch.as_tensor(np.asarray(m), device=self.mm.device, dtype=torch.float64).reshape(-1)[self._flat]
        return self.state

    def read_into(self, mm: Magnets, out: torch.Tensor):
        if mm is not self.mm:
            self.configure_for(mm)
        out.copy_(self.mm._m_dev.reshape(-1)[self._flat])


def _bins(n_bins, n_cells):
    """Bin of every cell along one axis: linspace(0, n_bins (1 - 1e-15), n_cells) as int
    (hotspice/io.py:350-351), and the half-open cell range of every bin."""
    b = np.linspace(0, n_bins * (1 - 1e-15), n_cells, dtype=int)
    lo = np.searchsorted(b, np.arange(n_bins), side='left')
    hi = np.searchsorted(b, np.arange(n_bins), side='right')
    return b, lo, hi


class _RegionReader(OutputReader):
    """Shared device readout over rectangular regions (hs_region_readout)."""

    def _setup_regions(self, mm, wx, wy, norm):
        bx, xlo, xhi = _bins(self.nx, mm.nx)
        by, ylo, yhi = _bins(self.ny, mm.ny)
        self.region = np.tile(bx, (mm.ny, 1)) + self.nx * np.tile(by, (mm.nx, 1)).T
        R = self.nx * self.ny
        rects = np.zeros((R, 4), dtype=np.int32)
        for r in range(R):
            ry, rx = divmod(r, self.nx)
            rects[r] = (ylo[ry], yhi[ry], xlo[rx], xhi[rx])
        dev = mm.device
        self._rects = torch.as_tensor(rects.reshape(-1), device=dev)
        self._wx = torch.as_tensor(wx, device=dev, dtype=torch.float64).contiguous()
        self._wy = None if wy is None else torch.as_tensor(wy, device=dev, dtype=torch.float64).contiguous()
        self._norm = torch.as_tensor(norm, device=dev, dtype=torch.float64)

    def _launch(self, m_dev, out):
        mm = self.mm
        _lib.check(mm._lib.hs_region_readout(m_dev.data_ptr(), mm.nx, mm.ny, self.nx * self.ny, self._rects.data_ptr(),
                                             self._wx.data_ptr(), None if self._wy is None else self._wy.data_ptr(),
                                             self._norm.data_ptr(), out.data_ptr(), mm._stream()), 'hs_region_readout')

    def read_state(self, mm: Magnets = None, m=None) -> torch.Tensor:
        super().read_state(mm)
        if self.mm is None:
            raise AttributeError("OutputReader has not yet been initialized with a Magnets object.")
        if m is None:
            m_dev = self.mm._m_dev
        else:
            m_dev = torch.as_tensor(np.sign(np.asarray(m, dtype=float)), device=self.mm.device).to(torch.int8).contiguous()
        out = torch.empty_like(self.state)
        self._launch(m_dev, out)
        self.state = out
        return self.state

    def read_into(self, mm: Magnets, out: torch.Tensor):
        if mm is not self.mm:
            self.configure_for(mm)
        self._launch(self.mm._m_dev, out)


class RegionalOutputReader(_RegionReader):
    """hotspice/io.py:335-379: nx x ny regions; per region the moment-weighted magnetisation
    (x and y components in plane), normalised by the region's total moment."""

    def __init__(self, nx: int, ny: int, mm: Magnets = None):
        self.nx, self.ny = nx, ny
        self.n_regions = self.nx * self.ny
        super().__init__(mm)

    def configure_for(self, mm: Magnets):
        self.mm = mm
        R = self.n_regions
        self.state = torch.zeros(R * 2 if mm.in_plane else R, device=mm.device, dtype=torch.float64)
        mom = np.asarray(mm._moment_np, dtype=float)
        occ = np.asarray(mm.occupation)
        if mm.in_plane:
            wx, wy = mom * mm.orientation[:, :, 0], mom * mm.orientation[:, :, 1]
        else:
            wx, wy = mom, None
        self._setup_regions(mm, wx, wy, np.zeros(1))
        n = self.state.numel()
        norm = np.zeros(n)
        self._node_coords = np.zeros((n, 2))
        for i in range(n):
            r = i % R
            sel = self.region == r
            norm[i] = np.sum(occ[sel] * mom[sel])
            self._node_coords[i, 0] = np.mean(mm.xx[sel])
            self._node_coords[i, 1] = np.mean(mm.yy[sel])
        self.normalization_factor = norm
        self._norm = torch.as_tensor(norm[:R], device=mm.device, dtype=torch.float64)


class OOPSquareChessOutputReader(_RegionReader):
    """hotspice/io.py:404-446: per region the checkerboard-masked magnetisation (distinguishes
    the two antiferromagnetic ground states of OOP_Square), normalised by the magnet count."""

    def __init__(self, nx: int, ny: int, mm: OOP_Square = None):
        self.nx, self.ny = int(nx), int(ny)
        super().__init__(mm)

    def configure_for(self, mm: OOP_Square):
        if not isinstance(mm, (expected_type := OOP_Square)):
            if mm.in_plane:
                raise TypeError(f"{type(self).__name__} only works on out-of-plane ASI, but received {type(mm).__name__}.")
            warnings.warn(f"{type(self).__name__} expects {expected_type.__name__} ASI, but received {type(mm).__name__}.", stacklevel=2)
        self.mm = mm
        R = self.nx * self.ny
        self.state = torch.zeros(R, device=mm.device, dtype=torch.float64)
        self.AFM_mask = ((mm.ixx + mm.iyy) % 2) * 2 - 1
        self._setup_regions(mm, self.AFM_mask.astype(float), None, np.zeros(1))
        norm = np.zeros(R, dtype=int)
        self._node_coords = np.zeros((R, 2))
        occ = np.asarray(mm.occupation)
        for r in range(R):
            sel = self.region == r
            norm[r] = np.sum(occ[sel])
            self._node_coords[r, 0] = np.mean(mm.xx[sel])
            self._node_coords[r, 1] = np.mean(mm.yy[sel])
        self.normalization_factor = norm
        self._norm = torch.as_tensor(norm.astype(float), device=mm.device, dtype=torch.float64)


# ------------------------------------------------------------------------------ sequences
def run_sequence(mm: Magnets, inputter: Inputter, values=None, reader: OutputReader = None, n: int = None):
    """Input every value of ``values`` (default: ``n`` values of the inputter's datastream)
    and read the state after each one: the loop of the reference's experiments
    (``inputter.input(mm, value)`` then ``reader.read_state()``), enqueued on the device
    without a host round trip per input. Returns (values, readouts) with readouts a
    (len(values), reader.n) float64 device tensor (None without a reader)."""
    if values is None:
        values = inputter.datastream.get_next(n=1 if n is None else n)
    values = np.asarray(values).reshape(-1)
    out = None
    if reader is not None:
        if reader.mm is not mm:
            reader.configure_for(mm)
        out = torch.empty((values.size, reader.n), device=mm.device, dtype=torch.float64)
    gen = isgeneratorfunction(inputter.input_single)
    for k, v in enumerate(values):
        for b in _expand(inputter, np.asarray([v])):
            result = inputter.input_single(mm, b)
            if gen:
                for _ in result:
                    pass
        if out is not None:
            reader.read_into(mm, out[k])
    mm._progress_finish()
    return values, out


def run_batch(mms, inputter: Inputter, values, readers=None):
    """Drive several reservoirs at once: instance i receives the sequence ``values[i]`` (or
    the shared 1-D ``values``) and is read by ``readers[i]`` after every input. Per input
    stage the fields and progress() stop rules of all instances are set on the device, then
    ONE persistent engine launch advances every instance until its own stop rule holds
    (instances are independent: each result equals its :func:`run_sequence`). The inputter
    must describe its inputs as stages (every input except the sinusoidal FieldInputter and
    PerpFieldInputter with relax=True). Returns a list of (len, reader.n) float64 device
    tensors (None without readers); synchronises once, at the end."""
    from .engine import BatchEngine
    mms = list(mms)
    M = len(mms)
    vals = np.asarray(values)
    vals = np.broadcast_to(vals, (M, vals.size)) if vals.ndim <= 1 else vals
    if vals.shape[0] != M:
        raise ValueError(f'values has {vals.shape[0]} rows for {M} instances')
    K = vals.shape[1]
    for mm in mms:
        _zeeman(mm)                     # before the launch descriptors are made
    outs = None
    if readers is not None:
        if len(readers) != M:
            raise ValueError('one reader per instance')
        for mm, rd in zip(mms, readers):
            if rd.mm is not mm:
                rd.configure_for(mm)
        outs = [torch.empty((K, rd.n), device=mm.device, dtype=torch.float64) for mm, rd in zip(mms, readers)]
    eng = BatchEngine(mms)
    prepared = eng._prepare([0] * M, [{} for _ in mms])
    for k in range(K):
        bits = [_expand(inputter, np.asarray([vals[i, k]])) for i in range(M)]
        for b in range(len(bits[0])):
            plans = [inputter.stages(mm, bits[i][b]) for i, mm in enumerate(mms)]
            if any(p is None for p in plans):
                raise NotImplementedError(f'{type(inputter).__name__} needs the host between steps: use run_sequence')
            for j in range(len(plans[0])):
                for mm, plan in zip(mms, plans):
                    st = plan[j]
                    mm.get_energy('Zeeman', verbose=False).set_field_device(st.magnitude, pattern=st.pattern, angle=st.angle)
                    mm._progress_arm(t_max=st.t_max, MCsteps_max=st.mc_max)
                eng.launch(prepared)
        if outs is not None:
            for i, (mm, rd) in enumerate(zip(mms, readers)):
                rd.read_into(mm, outs[i][k])
    for mm in mms:
        mm._progress_finish()
    return outs
