"""ctypes binding of libhotspice_sm100.so (C ABI in include/hotspice_b200.h).

The library is built in-tree (``python -m hotspice_b200.build``). There is no fallback:
if the library is missing or was built for another ABI, importing the engine raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, 'libhotspice_sm100.so')

HS_OK, HS_EINVAL, HS_ENOMEM, HS_ETIMEDOUT, HS_ECUDA, HS_ERANGE = 0, -1, -2, -3, -4, -5
HS_ST_SELECT_RETRY, HS_ST_SWITCH_OVERFLOW, HS_ST_POISSON_OVERFLOW, HS_ST_WOLFF_OVERFLOW, HS_ST_STEP_CAP = 1, 2, 4, 8, 16
HS_PROGRESS_STEPS_MAX = 1 << 22
HS_ENGINE_WS_DEFAULT, HS_ENGINE_WS_MAX = 64 * 1024, 160 * 1024
HS_SAMPLE_SINGLE, HS_SAMPLE_GRID, HS_SAMPLE_POISSON = 0, 1, 2
HS_BARRIER_SIMPLE, HS_BARRIER_PARABOLIC = 0, 1
HS_UPDATE_SINGLE, HS_UPDATE_MULTIPLE = 0, 1
HS_SEGMENT_MAX = 65536
HS_INST_ONE_CTA = 1   # HsInstance.flags: run on one CTA of its cluster

P = C.c_void_p


class HsLattice(C.Structure):
    _fields_ = [
        ('m', P), ('occ', P), ('mm', P), ('moment', P), ('nonzero', P), ('sub_of', P), ('E_B', P), ('beta', P),
        ('K', P), ('Kpo', P), ('Kps', P), ('E_dip', P), ('E_dip_perp', P), ('zee', P), ('zee_perp', P),
        ('orient', P), ('wolff_bond', P),
        ('beta_uniform', C.c_double), ('J', C.c_double), ('dip_pref', C.c_double), ('m_perp_factor', C.c_double),
        ('seed', C.c_uint64),
        ('nx', C.c_int32), ('ny', C.c_int32), ('ux', C.c_int32), ('uy', C.c_int32), ('pbc', C.c_int32),
        ('in_plane', C.c_int32), ('use_perp', C.c_int32), ('n_occ', C.c_int32), ('barrier_method', C.c_int32),
        ('has_dipolar', C.c_int32), ('dip_wx', C.c_int32), ('dip_wy', C.c_int32), ('dip_wrap', C.c_int32),
        ('n_sub', C.c_int32), ('has_exchange', C.c_int32), ('nn_h', C.c_int32), ('nn_w', C.c_int32),
        ('trunc_cutoff', C.c_int32), ('trunc_size', C.c_int32), ('dip_keep_perp_sign', C.c_int32),
        ('nn', C.c_int8 * 28),
    ]


class HsCounters(C.Structure):
    _fields_ = [
        ('t', C.c_double), ('t0', C.c_double), ('mc0', C.c_double), ('t_max', C.c_double), ('mc_max', C.c_double),
        ('switches', C.c_int64), ('attempted', C.c_int64), ('rng_call', C.c_uint64),
        ('status', C.c_int32), ('done', C.c_int32), ('progress', C.c_int32), ('n_sw', C.c_int32),
        ('epoch', C.c_int32), ('steps', C.c_int32),
        ('bmin', C.c_double), ('last_time', C.c_double), ('near_threshold', C.c_int64), ('reserved', C.c_double * 4),
    ]


class HsSwitchList(C.Structure):
    _fields_ = [('y', P), ('x', P), ('mode', P), ('cap', C.c_int32), ('pad', C.c_int32)]


class HsGridPlan(C.Structure):
    _fields_ = [
        ('phase_off', P), ('phase_yx', P), ('Rx', C.c_int32), ('Ry', C.c_int32), ('snx', C.c_int32),
        ('sny', C.c_int32), ('n_sc', C.c_int32), ('sample_scheme', C.c_int32), ('r_cells', C.c_double),
        ('poisson_k', C.c_int32), ('metropolis_time', C.c_int32), ('attempt_freq', C.c_double),
    ]


# numpy mirror of HsCounters, for device <-> host transfers of the raw bytes
COUNTERS_DTYPE = np.dtype({
    'names': [f[0] for f in HsCounters._fields_],
    'formats': ['<f8', '<f8', '<f8', '<f8', '<f8', '<i8', '<i8', '<u8', '<i4', '<i4', '<i4', '<i4', '<i4', '<i4',
                '<f8', '<f8', '<i8', ('<f8', (4,))],
    'offsets': [getattr(HsCounters, f[0]).offset for f in HsCounters._fields_],
    'itemsize': C.sizeof(HsCounters),
})

# symbol -> (restype, argtypes); every symbol include/hotspice_b200.h declares
SIGNATURES = {
    'hs_version': (C.c_int, []),
    'hs_last_error': (C.c_int, [C.c_char_p, C.c_int]),
    'hs_struct_sizes': (C.c_int, [C.POINTER(C.c_int32), C.c_int]),
    'hs_philox_uniform': (C.c_int, [C.c_uint64, C.c_uint64, C.c_int32, P, P]),
    'hs_dipolar_update': (C.c_int, [C.POINTER(HsLattice), C.POINTER(HsSwitchList), P, C.c_int32, C.c_int32, P, P]),
    'hs_dipolar_full_direct': (C.c_int, [C.POINTER(HsLattice), C.c_int32, P, P, P]),
    'hs_igemm_scratch_bytes': (C.c_int64, [C.POINTER(HsLattice), C.c_int32]),
    'hs_dipolar_full_igemm': (C.c_int, [C.POINTER(HsLattice), C.c_int32, P, C.c_int64, P]),
    'hs_set_wait_limit': (C.c_int, [C.c_uint64]),
    'hs_neel_scratch_bytes': (C.c_int64, [C.POINTER(HsLattice)]),
    'hs_neel_step': (C.c_int, [C.POINTER(HsLattice), P, C.POINTER(HsSwitchList), C.c_double, P, C.c_int64, P]),
    'hs_metropolis_scratch_bytes': (C.c_int64, [C.POINTER(HsLattice), C.POINTER(HsGridPlan)]),
    'hs_metropolis_step': (C.c_int, [C.POINTER(HsLattice), P, C.POINTER(HsSwitchList), C.POINTER(HsGridPlan), P,
                                     C.c_int64, P]),
    'hs_metropolis_step_noalloc': (C.c_int, [C.POINTER(HsLattice), P, C.POINTER(HsSwitchList),
                                             C.POINTER(HsGridPlan), P]),
    'hs_wolff_scratch_bytes': (C.c_int64, [C.POINTER(HsLattice)]),
    'hs_wolff_step': (C.c_int, [C.POINTER(HsLattice), P, C.POINTER(HsSwitchList), P, C.c_int64, P]),
    'hs_relax_scratch_bytes': (C.c_int64, [C.POINTER(HsLattice)]),
    'hs_relax_begin': (C.c_int, [C.POINTER(HsLattice), P, C.c_int64, P]),
    'hs_relax_permute': (C.c_int, [C.POINTER(HsLattice), P, C.c_int32, P, C.c_int64, P]),
    'hs_relax_subset': (C.c_int, [C.POINTER(HsLattice), P, C.POINTER(HsSwitchList), C.c_int32, C.c_int32, C.c_int32,
                                  P, C.c_int64, P]),
    'hs_minimize_all': (C.c_int, [C.POINTER(HsLattice), P, C.POINTER(HsSwitchList), C.c_int32, C.c_int32, P,
                                  C.c_int64, P]),
    'hs_relax_check': (C.c_int, [C.POINTER(HsLattice), P, C.c_int32, P, C.c_int64, P]),
    'hs_minimize_begin': (C.c_int, [C.POINTER(HsLattice), P, C.c_int64, P]),
    'hs_minimize_step': (C.c_int, [C.POINTER(HsLattice), P, C.POINTER(HsSwitchList), C.c_double, P, C.c_int64, P]),
    'hs_zeeman_set': (C.c_int, [C.c_int64, C.c_int32, P, P, P, C.c_double, C.c_double, P, P, P, P, P]),
    'hs_progress_arm': (C.c_int, [P, C.c_int32, C.c_double, C.c_double, P]),
    'hs_progress_disarm': (C.c_int, [P, P]),
    'hs_region_readout': (C.c_int, [P, C.c_int32, C.c_int32, C.c_int32, P, P, P, P, P, P]),
    'hs_square_vertex_counts': (C.c_int, [P, C.c_int32, C.c_int32, P, P]),
    'hs_segments_copy': (C.c_int, [P, P, C.c_int32, C.c_int32, P]),
    'hs_engine_run': (C.c_int, [P, C.c_int32, C.c_int32, C.c_int32, P, P]),
    'hs_engine_run_ws': (C.c_int, [P, C.c_int32, C.c_int32, C.c_int32, P, C.c_int32, P, P]),
    'hs_engine_max_clusters': (C.c_int, [C.c_int32]),
    'hs_exchange_energy': (C.c_int, [C.POINTER(HsLattice), P, P, P]),
    'hs_switch_energy': (C.c_int, [C.POINTER(HsLattice), P, P]),
}

_lib = None


def load():
    """Load and type the library (once). Raises if it is missing or its ABI differs."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f'{LIB_PATH} is missing: build it with `python -m hotspice_b200.build` '
                           '(hotspice_b200 has no CPU fallback)')
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    sizes = (C.c_int32 * 5)()
    lib.hs_struct_sizes(sizes, 5)
    want = [C.sizeof(HsLattice), C.sizeof(HsCounters), C.sizeof(HsSwitchList), C.sizeof(HsGridPlan),
            HsLattice.nx.offset]
    if list(sizes) != want:
        raise RuntimeError(f'ABI mismatch between {LIB_PATH} and hotspice_b200._lib: {list(sizes)} != {want}')
    _lib = lib
    return lib


def last_error() -> str:
    buf = C.create_string_buffer(512)
    load().hs_last_error(buf, 512)
    return buf.value.decode(errors='replace')


def check(rc: int, what: str = ''):
    if rc != HS_OK:
        msg = last_error()
        if rc == HS_EINVAL:
            raise ValueError(f'{what}: {msg}')
        raise RuntimeError(f'{what} failed ({rc}): {msg}')
    return rc
