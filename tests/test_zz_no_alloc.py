"""The allocation-free Metropolis entry point against the regular one.

hs_metropolis_step_noalloc serves callers that cannot allocate device memory (an embedding
application that only hands over its state arrays, or a loop that must never call
cudaMalloc): its working arrays live in a fixed 4 MiB device array inside the library
instead of a caller-provided scratch buffer. Two identical lattices are advanced, one
through each entry point via the C ABI, for two calls in a row; spins, energies, counters
and switch lists must agree exactly (same kernels, same variates, deterministic order).
"""
import ctypes

import numpy as np
import pytest

from gpu_cases import build_product

pytestmark = pytest.mark.gpu


def _state(mm):
    import torch
    d = mm.get_energy('dipolar')
    t, _ = mm._sw
    n = int(mm._read_counters()['n_sw'])
    return (mm._m_dev.cpu().numpy().copy(), d._E.cpu().numpy().copy(),
            d._Ep.cpu().numpy().copy() if d._Ep is not None else None,
            mm._read_counters().copy(), t[:2, :n].cpu().numpy().copy())


@pytest.mark.parametrize('name', ['metro_pin32_grid', 'metro_oop32_trunc_pbc'])
def test_noalloc_matches_regular_entry_point(name):
    import torch
    from cases import load_specs
    from hotspice_b200 import _lib
    lib = _lib.load()
    spec = load_specs()[name]
    r = spec['update_kw']['r']
    a = build_product(name)
    b = build_product(name)
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        kind, L, s, P, buf = a._step_args({'r': r})
        assert kind == 'metro'
        _lib.check(lib.hs_metropolis_step(L, a._counters.data_ptr(), s, P, buf.data_ptr(), buf.numel(), stream),
                   'hs_metropolis_step')
        kind, Lb, sb, Pb, _ = b._step_args({'r': r})
        _lib.check(lib.hs_metropolis_step_noalloc(Lb, b._counters.data_ptr(), sb, Pb, stream),
                   'hs_metropolis_step_noalloc')
        torch.cuda.synchronize()
        sa, sbb = _state(a), _state(b)
        assert np.array_equal(sa[0], sbb[0]), f'call {call}: spins differ'
        assert np.array_equal(sa[1], sbb[1]), f'call {call}: E differs'
        if sa[2] is not None:
            assert np.array_equal(sa[2], sbb[2]), f'call {call}: E_perp differs'
        for k in ('attempted', 'switches', 'rng_call', 'n_sw', 'status'):
            assert sa[3][k] == sbb[3][k], f'call {call}: counter {k} differs'
        assert np.array_equal(sa[4], sbb[4]), f'call {call}: switch lists differ'
        assert int(sa[3]['attempted']) > 0


def test_noalloc_rejects_plans_beyond_its_fixed_scratch():
    """A plan whose working arrays exceed the fixed 4 MiB is refused with HS_ERANGE."""
    from hotspice_b200 import _lib
    lib = _lib.load()
    a = build_product('metro_pin32_grid')
    kind, L, s, P, buf = a._step_args({'r': 4 * 300e-9})
    big = _lib.HsGridPlan()
    ctypes.memmove(ctypes.byref(big), ctypes.byref(P), ctypes.sizeof(P))
    big.n_sc = 1 << 20   # 8 MiB of candidate positions
    rc = lib.hs_metropolis_step_noalloc(L, a._counters.data_ptr(), s, big, None)
    assert rc == _lib.HS_ERANGE
    assert 'fixed scratch holds' in _lib.last_error()
