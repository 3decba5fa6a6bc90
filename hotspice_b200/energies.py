"""Energy plugins with the reference's interface (hotspice/energies.py:22-83), backed by
device buffers and the sm_100a kernels of libhotspice_sm100.so.

Contract kept from the reference:
* ``initialize(mm)`` -> ``_initialize()`` then ``update()``;
* ``update()`` is a full recompute; ``update_single(index2D)`` / ``update_multiple(indices2D)``
  are called *after* the spins at the indices were flipped (row 0 = y, row 1 = x);
* ``energy_switch(indices2D)`` = -2 E at the indices; properties ``E``, ``E_perp``, ``E_tot``.

``E`` / ``E_perp`` are returned as float64 torch tensors on the simulation's device. The
engine keeps the dipolar energy in float32 (incremental updates) and recomputes it in full
on demand (FP64 direct sum or the tensor-core implicit GEMM); the Zeeman and exchange
energies are evaluated from the spins when needed, which gives exactly the values the
reference's sign flips / recomputations produce.
"""
from __future__ import annotations

import math
from functools import cached_property

import numpy as np
import torch

from . import _lib
from .utils import copy_to_device, to_device
from .kernels import build_dimonopolar_kernels, build_kernels


class Energy:
    def __init__(self):
        pass

    def energy_switch(self, indices2D=None):
        """-2 E at ``indices2D`` (or everywhere), hotspice/energies.py:29-35."""
        E = self.E
        if indices2D is None:
            return -2 * E
        idx = torch.as_tensor(np.asarray(indices2D), device=E.device, dtype=torch.long)
        return -2 * E[idx[0], idx[1]]

    def initialize(self, mm):
        """(Re)bind to ``mm`` and recompute, hotspice/energies.py:37-42."""
        self.mm = mm
        self._initialize()
        self.update()

    def _initialize(self):
        pass

    def update(self):
        raise NotImplementedError

    def update_single(self, index2D):
        raise NotImplementedError

    def update_multiple(self, indices2D):
        raise NotImplementedError

    E_div = 1   # E_tot = E_sum() / E_div (2 for pair energies, counted once per pair)

    def E_sum(self) -> torch.Tensor:
        """The sum behind E_tot as a 0-d device tensor (read later without a host sync)."""
        raise NotImplementedError

    @property
    def E_tot(self):
        return float(self.E_sum()) / self.E_div

    @cached_property
    def shortname(self):
        return type(self).__name__.lower().replace('energy', '')


class ZeemanEnergy(Energy):
    """Uniform external field (hotspice/energies.py:86-140). E = m * E_factor."""

    def __init__(self, magnitude=0, angle=0):
        self._magnitude = magnitude
        self._angle = angle

    def _initialize(self):
        self.set_field(magnitude=self._magnitude, angle=self._angle)

    def set_field(self, magnitude=None, angle=None):
        if magnitude is None:
            self._resolve_lazy()
        self._lazy = None
        if magnitude is not None:
            self._magnitude = magnitude
        if angle is not None:
            self._angle = angle
        if not hasattr(self, 'mm'):
            return
        mm = self.mm
        mag = mm._field(self._magnitude)
        ang = mm._field(self._angle)
        mom = mm._moment_np
        if mm.in_plane:
            bx, by = mag * np.cos(ang), mag * np.sin(ang)
            o = mm.orientation
            ef = -mom * (bx * o[:, :, 0] + by * o[:, :, 1])
            efp = -mom * (by * o[:, :, 0] - bx * o[:, :, 1])
        else:
            ef = -mom * mag
            efp = np.zeros_like(ef)
        self.E_factor = to_device(ef, mm.device, torch.float64)
        self.E_factor_perp = to_device(efp, mm.device, torch.float64)
        self._ef32 = self.E_factor.float().contiguous()
        self._efp32 = self.E_factor_perp.float().contiguous()
        mm._state_changed()

    def update(self):
        pass  # evaluated from the spins

    def update_single(self, index2D):
        pass

    def update_multiple(self, indices2D):
        pass

    @property
    def E(self):
        return self.mm._m_dev.double() * self.E_factor

    @property
    def E_perp(self):
        if not self.mm.USE_PERP_ENERGY:
            return torch.zeros_like(self.E_factor)
        return self.mm._m_dev.double() * self.E_factor_perp

    def E_sum(self):
        return torch.sum(self.E)

    def set_field_device(self, magnitude: float, pattern: torch.Tensor | None = None, angle: float | None = None):
        """set_field(magnitude * pattern, angle) computed on the device into the existing
        buffers (hs_zeeman_set): stream-ordered, no host round trip, and the lattice struct and
        captured graphs that point at the buffers stay valid. ``pattern``: an FP32 (ny, nx)
        device tensor (None: uniform); ``angle`` None keeps the current (scalar) angle."""
        mm = self.mm
        if angle is not None:
            self._angle = float(angle)
        ang = self._angle
        if mm.in_plane and not np.isscalar(ang):
            a = np.asarray(ang, dtype=float)
            if a.size and np.all(a == a.flat[0]):
                ang = float(a.flat[0])
            else:
                raise NotImplementedError('set_field_device needs a uniform angle')
        self._lazy = (float(magnitude), pattern)
        _lib.check(mm._lib.hs_zeeman_set(mm.nx * mm.ny, int(mm.in_plane), mm._moment64().data_ptr(),
                                         mm._orient64().data_ptr() if mm.in_plane else None,
                                         pattern.data_ptr() if pattern is not None else None, float(magnitude),
                                         float(ang) if mm.in_plane else 0.0, self.E_factor.data_ptr(),
                                         self.E_factor_perp.data_ptr(), self._ef32.data_ptr(), self._efp32.data_ptr(),
                                         mm._stream()), 'hs_zeeman_set')

    def _resolve_lazy(self):
        """Turn a magnitude set on the device back into the host-side value."""
        lz = getattr(self, '_lazy', None)
        if lz is not None:
            self._lazy = None
            scale, pat = lz
            self._magnitude = scale if pat is None else pat.double().cpu().numpy() * scale

    @property
    def magnitude(self):
        lz = getattr(self, '_lazy', None)
        if lz is not None:
            scale, pat = lz
            return self.mm._field(scale if pat is None else pat.double().cpu().numpy() * scale)
        return self.mm._field(self._magnitude)

    @magnitude.setter
    def magnitude(self, value):
        self.set_field(magnitude=value)

    @property
    def angle(self):
        return self.mm._field(self._angle)

    @angle.setter
    def angle(self, value):
        self.set_field(angle=value)


class DipolarEnergy(Energy):
    """Magnetostatic interaction between the magnets (hotspice/energies.py:143-391)."""

    def __init__(self, prefactor: float = 1, decay_exponent: float = -3, cutoff_range: float = math.inf):
        self._prefactor = prefactor
        self.decay_exponent = decay_exponent
        self._cutoff_range = cutoff_range

    @property
    def prefactor(self):
        return self._prefactor

    @prefactor.setter
    def prefactor(self, value):
        if hasattr(self, '_E'):
            self._E.mul_(value / self._prefactor)
            if self._Ep is not None:
                self._Ep.mul_(value / self._prefactor)
        self._prefactor = value
        if hasattr(self, 'mm'):
            self.mm._state_changed()

    @property
    def cutoff_range(self):
        return self._cutoff_range

    @cutoff_range.setter
    def cutoff_range(self, value):
        self._cutoff_range = value
        if hasattr(self, 'mm'):
            self._initialize()
            self.update()

    # DiMonopolarEnergy.update_multiple leaves E_perp of the switched magnets as it is
    # (hotspice/energies.py:718-719); DipolarEnergy.update_multiple negates it (334).
    _keep_perp_sign = False

    def _initialize(self):
        self._install(build_kernels(self.mm, self._cutoff_range, self.decay_exponent))

    def _install(self, ks):
        """Upload the kernels of ``ks`` and allocate the FP64 energy accumulators."""
        mm = self.mm
        self.kernel_set = ks
        dev = mm.device
        self._K = to_device(ks.K, dev, torch.float32)
        self._Kpo = to_device(ks.Kpo, dev, torch.float32) if mm.in_plane else None
        self._Kps = to_device(ks.Kps, dev, torch.float32) if mm.in_plane else None
        self._sub_of = to_device(ks.sub_of.reshape(-1), dev, torch.int32)
        self.kernel_unitcell_indices = ks.sub_of
        # FP64 accumulators of the FP32 per-switch increments (see hs_dipolar.cu)
        self._E = torch.zeros((mm.ny, mm.nx), device=dev, dtype=torch.float64)
        self._Ep = torch.zeros_like(self._E) if mm.in_plane else None
        mm._state_changed()

    @property
    def unitcell(self):
        return self.mm.unitcell

    def update(self, method: str | None = None):
        """Full recompute (hotspice/energies.py:290-308). ``method``: 'direct64' (FP64
        direct sum, the default up to EngineConfig.direct_max_pairs cell pairs), 'direct32',
        or 'igemm' (split-BF16 tensor-core implicit GEMM)."""
        self.mm._full_recompute(self, method)

    def update_single(self, index2D):
        self.mm._dipolar_apply(self, index2D, _lib.HS_UPDATE_SINGLE)

    def update_multiple(self, indices2D):
        self.mm._dipolar_apply(self, indices2D, _lib.HS_UPDATE_MULTIPLE)

    @property
    def E(self):
        return self._E.clone()

    @E.setter
    def E(self, value):
        self._E.copy_(torch.as_tensor(value, device=self._E.device).reshape(self._E.shape))

    @property
    def E_perp(self):
        if self._Ep is None or not self.mm.USE_PERP_ENERGY:
            return torch.zeros_like(self._E, dtype=torch.float64)
        return self._Ep.clone()

    E_div = 2

    def E_sum(self):
        return torch.sum(self._E)

    def get_NN_interaction(self):
        """Largest nearest-neighbour kernel magnitude times prefactor * <moment>^2
        (hotspice/energies.py:372-387)."""
        ks = self.kernel_set
        NN = np.asarray(self.mm._get_nearest_neighbors())
        hy, hx = NN.shape[0] // 2, NN.shape[1] // 2
        largest = 0.0
        for k in ks.K:
            cy, cx = ks.wy, ks.wx
            win = k[cy - hy:cy + hy + 1, cx - hx:cx + hx + 1]
            largest = max(largest, float(np.max(np.abs(win * NN))))
        return largest * self.prefactor * self.mm.moment_avg ** 2

    def set_NN_interaction(self, value):
        self.prefactor = value / self.get_NN_interaction()


class DiMonopolarEnergy(DipolarEnergy):
    """Magnetostatic interaction with every magnet a pair of opposite magnetic charges
    q = moment / d a distance d apart along its axis (hotspice/energies.py:394-751).

    E_i = prefactor * q_i^2 * m_i * sum_j K_s(i)(j - i) m_j with the monopole-pair kernels of
    :func:`hotspice_b200.kernels.build_dimonopolar_kernels`. For a uniform moment mu and
    spacing d this is the dipolar update with the device field mm = m * mu and the kernels
    scaled by q^2 / mu^2 = 1 / d^2, so the same sm_100a kernels (incremental update, direct
    and tensor-core recompute, engine) run it unchanged. Two reference details are kept:
    q^2 is fixed when the energy is initialised (a later change of the moment does not change
    it, so the device kernels are rescaled by q^2 / mu_new^2), and an update of more than one
    switch leaves E_perp of the switched magnets unnegated.

    Supported: in-plane lattices (the reference reads ``original_angles``, which only in-plane
    lattices have), a uniform moment on the occupied cells and a scalar (or uniform) ``d``;
    anything else raises NotImplementedError."""

    _keep_perp_sign = True

    def __init__(self, prefactor=1, d=200e-9, small_d=200e-9):
        self._prefactor = prefactor
        self.d = d
        self.small_d = small_d

    @staticmethod
    def _uniform(values, what):
        v = np.asarray(values, dtype=float)
        if v.size == 0 or not np.all(v == v.flat[0]):
            raise NotImplementedError(f'DiMonopolarEnergy on the sm_100a path needs a uniform {what}')
        return float(v.flat[0])

    def _moment(self):
        mm = self.mm
        return self._uniform(np.asarray(mm._moment_np)[np.asarray(mm.occupation) != 0], 'moment')

    def _initialize(self):
        mm = self.mm
        d = self._uniform(self.d, 'monopole spacing d')
        mu = self._moment()
        self._charge_sq = (mu / d) ** 2          # energies.py:414-415, fixed from here on
        ks = build_dimonopolar_kernels(mm, d, self.small_d, scale=1.0)
        self._K_phys = ks
        self._mu_kernels = mu
        self._install(self._scaled(ks, self._charge_sq / mu ** 2))

    @staticmethod
    def _scaled(ks, f):
        from dataclasses import replace
        return replace(ks, K=ks.K * f, Kps=ks.Kps * f, Kpo=ks.Kpo * f)

    def _moment_changed(self):
        """The magnets' moment changed: keep q^2 from the initialisation (as the reference
        does) by rescaling the device kernels to q^2 / mu_new^2. The energies are not
        recomputed (the reference's are not either)."""
        mu = self._moment()
        if mu == self._mu_kernels:
            return
        ks = self._scaled(self._K_phys, self._charge_sq / mu ** 2)
        self.kernel_set = ks
        dev = self.mm.device
        copy_to_device(self._K, ks.K)
        if self._Kpo is not None:
            copy_to_device(self._Kpo, ks.Kpo)
            copy_to_device(self._Kps, ks.Kps)
        self._mu_kernels = mu
        self.mm._state_changed()

    @property
    def charge(self):
        """q = moment / d [A m] (energies.py:414), as fixed at initialisation."""
        return torch.full((self.mm.ny, self.mm.nx), math.sqrt(self._charge_sq), device=self.mm.device, dtype=torch.float64)

    @property
    def charge_sq(self):
        return torch.full((self.mm.ny, self.mm.nx), self._charge_sq, device=self.mm.device, dtype=torch.float64)

    @property
    def kernel_unitcell(self):
        """The monopole-pair kernels in J / (A m)^2 * m, as the reference stores them."""
        return self._K_phys.K

    @property
    def kernel_perpself_unitcell(self):
        return self._K_phys.Kps

    @property
    def kernel_perpother_unitcell(self):
        return self._K_phys.Kpo

    def get_NN_interaction(self):
        """hotspice/energies.py:372-387 as inherited by the reference's DiMonopolarEnergy: the
        largest nearest-neighbour kernel entry times prefactor * <moment>^2."""
        ks = self._K_phys
        NN = np.asarray(self.mm._get_nearest_neighbors())
        hy, hx = NN.shape[0] // 2, NN.shape[1] // 2
        largest = 0.0
        for k in ks.K:
            win = k[ks.wy - hy:ks.wy + hy + 1, ks.wx - hx:ks.wx + hx + 1]
            largest = max(largest, float(np.max(np.abs(win * NN))))
        return largest * self.prefactor * self.mm.moment_avg ** 2


class ExchangeEnergy(Energy):
    """Nearest-neighbour exchange (hotspice/energies.py:754-791), evaluated from the spins."""

    def __init__(self, J=1):
        self._J = J

    @property
    def J(self):
        return self._J

    @J.setter
    def J(self, value):
        self._J = value
        if hasattr(self, 'mm'):
            self.mm._state_changed()

    def _initialize(self):
        self.local_interaction = np.asarray(self.mm._get_nearest_neighbors())
        self.mm._state_changed()

    def update(self):
        pass

    def update_single(self, index2D):
        pass

    def update_multiple(self, indices2D):
        pass

    def _fields(self):
        mm = self.mm
        E = torch.empty((mm.ny, mm.nx), device=mm.device, dtype=torch.float32)
        Ep = torch.empty_like(E) if mm.in_plane else None
        L = mm._lattice_struct()
        _lib.check(_lib.load().hs_exchange_energy(L, E.data_ptr(), Ep.data_ptr() if Ep is not None else None,
                                                  mm._stream()), 'hs_exchange_energy')
        return E, Ep

    @property
    def E(self):
        return self._fields()[0].double()

    @property
    def E_perp(self):
        E, Ep = self._fields()
        if Ep is None or not self.mm.USE_PERP_ENERGY:
            return torch.zeros_like(E, dtype=torch.float64)
        return Ep.double()

    E_div = 2

    def E_sum(self):
        return torch.sum(self.E)
