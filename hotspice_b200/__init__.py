"""hotspice_b200: the kinetic Monte Carlo hot path of Hotspice on NVIDIA B200 (sm_100a).

Drop-in for ``hotspice.Magnets`` / ``SimParams`` / ``Scheme`` and the ``DipolarEnergy``,
``DiMonopolarEnergy``, ``ZeemanEnergy`` and ``ExchangeEnergy`` plugins:
``import hotspice_b200 as hotspice``.
The host layer is Python over torch CUDA tensors; the hot path is hand-written CUDA in
``libhotspice_sm100.so`` (C ABI: include/hotspice_b200.h), loaded through ctypes.
"""
from . import config
from .core import EngineConfig, Magnets, Scheme, SimParams, Unitcell, kB
from .energies import DiMonopolarEnergy, DipolarEnergy, Energy, ExchangeEnergy, ZeemanEnergy
from . import energies, utils
from . import ASI
from . import io

__all__ = ['ASI', 'config', 'energies', 'io', 'utils', 'kB', 'SimParams', 'Magnets', 'Scheme', 'EngineConfig',
           'Unitcell', 'Energy', 'ZeemanEnergy', 'DipolarEnergy', 'DiMonopolarEnergy', 'ExchangeEnergy']
