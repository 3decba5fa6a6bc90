"""Tensor-core implicit-GEMM recompute (hs_dipolar_full_igemm) against the FP64 direct sum.

The direct sum (dip_full_direct_kernel, FP64) is itself pinned to the oracle's FFT
convolution in test_gpu_parity.py; here the split-BF16 GEMM must reproduce it to the stated
relative tolerance (max |E_igemm - E_fp64| / max |E_fp64|) on lattices that exercise every
path of the tiling: one and several 128-column tiles, one and several 256-row tiles, ragged
edges, several sublattices with empty cells, periodic (folded) kernels and the
perpendicular energy.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = {3: 1e-6,      # 3 BF16 splits (the default): FP64 near field, FP32 chunks of the far field
       2: 2e-6}      # 2 splits: 16-bit kernel terms in the far field
TOL_SPLIT1 = 1e-2    # plain BF16 kernel (8-bit significand)


def _make(kind, n, ny=None, PBC=False, seed=5, monopoles=False):
    import hotspice_b200 as hs
    cls = {'oop': hs.ASI.OOP_Square, 'pin': hs.ASI.IP_Pinwheel, 'kag': hs.ASI.IP_Kagome,
           'sq': hs.ASI.IP_Square}[kind]
    a = {'oop': 200e-9, 'pin': 300e-9, 'kag': 500e-9, 'sq': 300e-9}[kind]
    kw = dict(nx=n, ny=ny) if ny is not None else dict(n=n)
    mm = cls(a, **kw, T=300, E_B=5e-20, moment=1e-15, pattern='random', PBC=PBC, seed=seed,
             energies=[hs.DiMonopolarEnergy(d=0.4 * a, small_d=0.15 * a) if monopoles else hs.DipolarEnergy()])
    return mm


def _compare(mm, nsplit=3):
    d = mm._dipolar()
    d.update(method='direct64')
    E0, Ep0 = d.E, d.E_perp
    mm.engine.igemm_splits = nsplit
    d.update(method='igemm')
    E1, Ep1 = d.E, d.E_perp
    torch.cuda.synchronize()
    scale = float(E0.abs().max())
    err = float((E1 - E0).abs().max()) / scale
    errp = 0.0
    if mm.USE_PERP_ENERGY:
        errp = float((Ep1 - Ep0).abs().max()) / max(float(Ep0.abs().max()), 1e-300)
    return err, errp


@pytest.mark.parametrize('kind,n,ny,PBC', [
    ('oop', 16, None, False),      # one tile, mostly padding
    ('oop', 12, 9, True),          # folded periodic kernel, odd sizes
    ('oop', 300, 270, False),      # 3 x 2 tiles, ragged edges
    ('oop', 128, 256, False),      # exactly one tile
    ('oop', 129, 257, True),       # one past a tile boundary in both directions
    ('pin', 40, None, False),      # two sublattices, perpendicular energy
    ('kag', 36, None, False),      # empty cells, several sublattices
    ('sq', 150, None, True),       # in-plane, periodic, two column tiles
])
@pytest.mark.parametrize('nsplit', [2, 3])
def test_igemm_matches_fp64(kind, n, ny, PBC, nsplit):
    mm = _make(kind, n, ny, PBC)
    err, errp = _compare(mm, nsplit)
    print(f'{kind} {mm.nx}x{mm.ny} PBC={PBC} nsplit={nsplit}: rel err {err:.2e} perp {errp:.2e}')
    assert err <= TOL[nsplit]
    assert errp <= TOL[nsplit]


@pytest.mark.parametrize('kind,n,PBC', [('pin', 96, False), ('kag', 40, True), ('sq', 130, False)])
def test_igemm_monopole_kernels(kind, n, PBC):
    """DiMonopolarEnergy runs through the same GEMM (kernels scaled by 1/d^2)."""
    mm = _make(kind, n, PBC=PBC, monopoles=True)
    err, errp = _compare(mm, 3)
    print(f'monopoles {kind} {mm.nx}x{mm.ny} PBC={PBC}: rel err {err:.2e} perp {errp:.2e}')
    assert err <= TOL[3] and errp <= TOL[3]


def test_igemm_split_levels():
    mm = _make('oop', 64)
    e1, _ = _compare(mm, 1)
    e2, _ = _compare(mm, 2)
    e3, _ = _compare(mm, 3)
    # with two or more splits the kernel is carried to 16+ bits and the FP32 accumulation
    # of the far field dominates, so splits 2 and 3 agree to within that error
    assert e1 <= TOL_SPLIT1
    assert max(e2, e3) < e1
    assert e2 <= TOL[2] and e3 <= TOL[3]


def test_igemm_energy_total():
    """Total dipolar energy to 1e-6 relative on a 512^2 lattice."""
    mm = _make('oop', 512, seed=11)
    d = mm._dipolar()
    d.update(method='direct64')
    e0 = d.E_tot
    d.update(method='igemm')
    e1 = d.E_tot
    assert abs(e1 - e0) <= 1e-6 * abs(e0)


def test_igemm_rejects_cropped_kernel():
    import hotspice_b200 as hs
    mm = hs.ASI.OOP_Square(200e-9, 32, T=300, E_B=5e-20, moment=1e-15, pattern='random', seed=1,
                           energies=[hs.DipolarEnergy(cutoff_range=4 * 200e-9)])
    with pytest.raises(ValueError):
        mm._dipolar().update(method='igemm')


def test_igemm_rejects_nonuniform_moment():
    mm = _make('oop', 32)
    mom = np.full((mm.ny, mm.nx), 1e-15)
    mom[3, 4] = 2e-15
    mm.moment = mom
    with pytest.raises(ValueError):
        mm._dipolar().update(method='igemm')


def test_igemm_wait_limit_runs_out_cleanly():
    """A pipeline wait that runs out ends the recompute cleanly: with the limit shortened to 1 us
    (hs_set_wait_limit) the epilogue's first wait for an accumulator chunk gives up, the call's
    status word carries bit 0 (the host raises), the kernel's copies land, its MMAs finish and
    TMEM is freed; with the default limit restored the next recompute on the same context is
    correct."""
    from hotspice_b200 import _lib
    lib = _lib.load()
    mm = _make('oop', 300, 270)
    d = mm._dipolar()
    try:
        assert lib.hs_set_wait_limit(1000) == _lib.HS_OK
        with pytest.raises(RuntimeError, match='status 1'):
            d.update(method='igemm')
    finally:
        lib.hs_set_wait_limit(0)
    torch.cuda.synchronize()
    err, _ = _compare(mm, 3)
    assert err <= TOL[3]
