"""CPU tests of the host-side logic: kernel windows, selection plans, the C ABI surface."""
import ctypes
import math
import os
import re
from types import SimpleNamespace

import numpy as np
import pytest

from cases import load_fixture, load_specs, oracle_geometry, rel_err

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SPECS = load_specs()


def _mock(spec, fx):
    from oracle.geometry import unitcell
    g = oracle_geometry(spec)
    ux, uy = unitcell(g)
    return SimpleNamespace(nx=g.nx, ny=g.ny, unitcell=SimpleNamespace(x=ux, y=uy), dx=g.dx, dy=g.dy,
                           orientation=g.orientation, occupation=g.occupation, in_plane=g.in_plane,
                           PBC=bool(fx['PBC']), major_axis=0.0, minor_axis=0.0)


def expand_window(ks, nx, ny, K):
    """Rebuild the full (2ny-1, 2nx-1) kernel from a device window, with the same rules as
    hs_kval in hotspice_b200/csrc/hs_common.cuh (crop, minimum-image wrap)."""
    out = np.zeros((K.shape[0], 2 * ny - 1, 2 * nx - 1))
    for p in range(2 * ny - 1):
        for q in range(2 * nx - 1):
            dy, dx = p - (ny - 1), q - (nx - 1)
            if ks.wrap:  # minimum image, as hs_minimage
                dy = dy % ny if (dy % ny) * 2 < ny else dy % ny - ny
                dx = dx % nx if (dx % nx) * 2 < nx else dx % nx - nx
            if abs(dy) <= ks.wy and abs(dx) <= ks.wx:
                out[:, p, q] = K[:, dy + ks.wy, dx + ks.wx]
    return out


@pytest.mark.parametrize('name', [n for n in SPECS if any(e['type'] == 'dipolar' for e in SPECS[n]['energies'])])
def test_kernel_windows_match_reference(name):
    from hotspice_b200.kernels import build_kernels
    spec, fx = SPECS[name], load_fixture(name)
    mm = _mock(spec, fx)
    cut = [e.get('cutoff', np.inf) for e in spec['energies'] if e['type'] == 'dipolar'][0]
    ks = build_kernels(mm, cut)
    assert np.array_equal(ks.sub_of, fx['kernel_index'])
    for win, ref in ((ks.K, fx['kernels']), (ks.Kps, fx['kernels_perpself']), (ks.Kpo, fx['kernels_perpother'])):
        full = expand_window(ks, mm.nx, mm.ny, win)
        assert rel_err(full, ref) < 1e-12, name
    if np.isfinite(cut):
        assert ks.wy < mm.ny - 1 or ks.wx < mm.nx - 1 or not ks.wrap


@pytest.mark.parametrize('name', [n for n in SPECS if any(e['type'] == 'dimonopolar' for e in SPECS[n]['energies'])])
def test_dimonopolar_kernels_match_reference(name):
    """The monopole-pair kernels (built on each centre's window) against the reference's
    full-grid construction; unoccupied cells carry angle 0 in the geometry, which the
    occupation mask makes irrelevant."""
    from hotspice_b200.kernels import build_dimonopolar_kernels
    spec, fx = SPECS[name], load_fixture(name)
    mm = _mock(spec, fx)
    mm.original_angles = oracle_geometry(spec).angles
    e = [e for e in spec['energies'] if e['type'] == 'dimonopolar'][0]
    ks = build_dimonopolar_kernels(mm, e['d'], e['small_d'])
    assert np.array_equal(ks.sub_of, fx['kernel_index'])
    assert ks.full and not ks.wrap and (ks.wy, ks.wx) == (mm.ny - 1, mm.nx - 1)
    for win, ref in ((ks.K, fx['kernels']), (ks.Kps, fx['kernels_perpself']), (ks.Kpo, fx['kernels_perpother'])):
        assert win.shape == ref.shape
        assert rel_err(win, ref) < 1e-15, name
    scaled = build_dimonopolar_kernels(mm, e['d'], e['small_d'], scale=1 / e['d'] ** 2)
    assert rel_err(scaled.K * e['d'] ** 2, fx['kernels']) < 1e-15


@pytest.mark.parametrize('kind,n,PBC,cut_a', [('oop', 40, False, 6), ('oop', 40, True, 6), ('pin', 48, False, 8),
                                              ('pin', 48, True, 8), ('kag', 40, False, 3), ('kag', 44, True, 3)])
def test_windowed_kernels_equal_full_construction(kind, n, PBC, cut_a):
    """With a finite cutoff the kernels are built on the cutoff window only; every entry must
    be the same bits as in the full (2ny-1, 2nx-1) construction, which builds the distances
    from the same full-range cumulative sums."""
    import hotspice_b200.kernels as KM
    from oracle import geometry as G
    from oracle.geometry import unitcell
    a = 300e-9
    g = {'oop': G.oop_square, 'pin': G.ip_pinwheel, 'kag': G.ip_kagome}[kind](a, n, PBC=PBC) if kind == 'kag' \
        else {'oop': G.oop_square, 'pin': G.ip_pinwheel}[kind](a, n)
    ux, uy = unitcell(g)
    mm = SimpleNamespace(nx=g.nx, ny=g.ny, unitcell=SimpleNamespace(x=ux, y=uy), dx=g.dx, dy=g.dy,
                         orientation=g.orientation, occupation=g.occupation, in_plane=g.in_plane, PBC=PBC,
                         major_axis=0.0, minor_axis=0.0)
    cut = cut_a * a
    ks = KM.build_kernels(mm, cut)
    dxc, dyc = np.asarray(g.dx[:ux], float), np.asarray(g.dy[:uy], float)
    ori = g.orientation[:uy, :ux] if g.in_plane else None
    occ = g.occupation[:uy, :ux]
    for y in range(uy):
        for x in range(ux):
            if ks.sub_of[y, x] < 0:
                continue
            full = KM._site_kernels(g.nx, g.ny, ux, uy, y, x, dxc, dyc, ori, occ, g.in_plane, cut, -3, 0.0)
            win = KM._site_kernels(g.nx, g.ny, ux, uy, y, x, dxc, dyc, ori, occ, g.in_plane, cut, -3, 0.0,
                                   (ks.wy, ks.wx))
            for f, w in zip(full, win):
                assert np.array_equal(f[g.ny - 1 - ks.wy:g.ny + ks.wy, g.nx - 1 - ks.wx:g.nx + ks.wx], w)
                # nothing non-zero outside the window
                mask = np.ones_like(f, dtype=bool)
                mask[g.ny - 1 - ks.wy:g.ny + ks.wy, g.nx - 1 - ks.wx:g.nx + ks.wx] = False
                assert not np.any(f[mask])
            s = ks.sub_of[y, x]
            assert np.array_equal(full[0][g.ny - 1 - ks.wy:g.ny + ks.wy, g.nx - 1 - ks.wx:g.nx + ks.wx] * 1e-7, ks.K[s])


def test_pbc_cutoff_window_is_minimum_image():
    """With PBC and a cutoff below half the lattice the stored window is unfolded and
    applied with wrapping; it must reproduce the folded kernel entry by entry."""
    from hotspice_b200.kernels import build_kernels
    from oracle.geometry import oop_square
    from oracle.hotspice_oracle import build_dipolar_kernels
    g = oop_square(1e-6, 24, 20)
    mm = SimpleNamespace(nx=24, ny=20, unitcell=SimpleNamespace(x=1, y=1), dx=g.dx, dy=g.dy, orientation=None,
                         occupation=g.occupation, in_plane=False, PBC=True, major_axis=0.0, minor_axis=0.0)
    ks = build_kernels(mm, cutoff=4.5e-6)
    assert ks.wrap and ks.wx == 4 and ks.wy == 4
    om = SimpleNamespace(**vars(mm))
    om.unitcell = (1, 1)
    K, _, _, _ = build_dipolar_kernels(om, 4.5e-6)
    assert rel_err(expand_window(ks, 24, 20, ks.K), K) < 1e-12


@pytest.mark.parametrize('name', ['metro_pin32_grid', 'metro_pin24_pbc', 'metro_kagome_grid', 'metro_oop30_trunc'])
def test_grid_plan_matches_oracle(name):
    """Supercell sizes of the device plan equal the oracle's (hotspice/core.py:509-516)."""
    from cases import build_oracle
    spec = SPECS[name]
    mm = build_oracle(name)
    r = spec['update_kw']['r']
    Rx, Ry, snx, sny = mm.grid_geometry(r)
    ux, uy = mm.unitcell
    Rx2 = max(min(ux * math.ceil((math.ceil(r / np.min(mm.dx)) - 1) / ux), mm.nx), 2)
    assert Rx2 == Rx
    n_sc = len(range(0, min(snx, mm.nx), 2)) * len(range(0, min(sny, mm.ny), 2))
    ixx = np.meshgrid(np.arange(mm.nx), np.arange(mm.ny))[0]
    assert n_sc == ixx[:sny:2, :snx:2].size


def test_library_exports_every_declared_symbol():
    from hotspice_b200 import _lib
    header = open(os.path.join(ROOT, 'include', 'hotspice_b200.h')).read()
    declared = set(re.findall(r'^\s*(?:int|int64_t)\s+(hs_\w+)\s*\(', header, flags=re.M))
    assert declared, 'no declarations parsed'
    lib = _lib.load()
    for name in declared:
        assert hasattr(lib, name), name
    assert declared <= set(_lib.SIGNATURES)
    assert lib.hs_version() == 1


def test_abi_struct_layout():
    from hotspice_b200 import _lib
    lib = _lib.load()
    sizes = (ctypes.c_int32 * 5)()
    lib.hs_struct_sizes(sizes, 5)
    assert list(sizes) == [ctypes.sizeof(_lib.HsLattice), ctypes.sizeof(_lib.HsCounters),
                           ctypes.sizeof(_lib.HsSwitchList), ctypes.sizeof(_lib.HsGridPlan), _lib.HsLattice.nx.offset]
    assert _lib.COUNTERS_DTYPE.itemsize == ctypes.sizeof(_lib.HsCounters)


def test_argument_validation_without_gpu():
    """Bad arguments are rejected on the host before any launch."""
    from hotspice_b200 import _lib
    lib = _lib.load()
    L = _lib.HsLattice()
    assert lib.hs_neel_step(ctypes.byref(L), None, None, 1e10, None, 0, None) == _lib.HS_EINVAL
    assert 'bad lattice size' in _lib.last_error()
    assert lib.hs_philox_uniform(1, 0, -1, None, None) == _lib.HS_EINVAL


def test_simparams_validation():
    from hotspice_b200 import Scheme, SimParams
    assert SimParams(UPDATE_SCHEME='Néel').UPDATE_SCHEME == Scheme.NEEL
    assert SimParams(UPDATE_SCHEME='Glauber').UPDATE_SCHEME == Scheme.METROPOLIS
    with pytest.raises(ValueError):
        SimParams(UPDATE_SCHEME='Gibbs')
    with pytest.raises(ValueError):
        SimParams(MULTISAMPLING_SCHEME='hex')


def test_lower_than_matches_reference_rule():
    from hotspice_b200.utils import lower_than
    from oracle.hotspice_oracle import lower_than as ref
    for x, y in [(1.0, 2.0), (1.0, 1.0 + 1e-11), (1 - 1e-12, 1.0), (2.0, 1.0), (0.0, 0.0), (-1.0, 0.0), (0.0, float('inf')),
                 (float('inf'), float('inf')), (1.0, -float('inf'))]:
        assert lower_than(x, y) == ref(x, y)


def test_truncated_window_sum_matches_convolve2d():
    """The oracle's scatter restatement of the >20-switch branch equals SciPy's
    convolve2d(..., 'same', wrap|fill) (hotspice/energies.py:345-350)."""
    from scipy import signal
    from oracle.hotspice_oracle import truncated_window_sum
    rng = np.random.default_rng(3)
    for PBC in (False, True):
        for ny, nx, R in ((30, 26, 20), (12, 9, 20), (40, 44, 5)):
            K = rng.normal(size=(2 * ny - 1, 2 * nx - 1))
            mmom = rng.choice([-1.0, 1.0], size=(ny, nx)) * 1.3
            here = np.asarray(np.nonzero(rng.random((ny, nx)) < 0.1))
            mm = SimpleNamespace(ny=ny, nx=nx, PBC=PBC, params={'REDUCED_KERNEL_SIZE': R}, m=mmom)
            got = truncated_window_sum(mm, here, mmom, K)
            sf = np.zeros((ny, nx))
            sf[here[0], here[1]] = mmom[here[0], here[1]]
            kx, ky = min(R, nx - 1), min(R, ny - 1)
            crop = K[ny - 1 - ky:ny + ky, nx - 1 - kx:nx + kx]
            ref = signal.convolve2d(sf, crop, mode='same', boundary='wrap' if PBC else 'fill')
            assert np.allclose(got, ref, rtol=1e-12, atol=1e-12)


def test_new_entry_points_reject_bad_arguments_without_a_launch():
    """The relaxation, reservoir I/O and packed-transfer entry points validate their arguments on
    the host and return HS_EINVAL before any launch (so this runs without a GPU)."""
    import ctypes as C
    from hotspice_b200 import _lib
    lib = _lib.load()
    L, sw = _lib.HsLattice(), _lib.HsSwitchList()
    assert lib.hs_segments_copy(None, None, -1, 1, None) == _lib.HS_EINVAL
    assert lib.hs_segments_copy(None, None, 0, 1, None) == _lib.HS_OK          # nothing to move
    assert lib.hs_region_readout(None, 4, 4, 1, None, None, None, None, None, None) == _lib.HS_EINVAL
    assert lib.hs_zeeman_set(0, 0, None, None, None, 1.0, 0.0, None, None, None, None, None) == _lib.HS_EINVAL
    assert lib.hs_progress_arm(None, 1, 1.0, 1.0, None) == _lib.HS_EINVAL
    assert lib.hs_progress_disarm(None, None) == _lib.HS_EINVAL
    assert lib.hs_relax_scratch_bytes(C.byref(L)) == -1                          # empty lattice
    assert lib.hs_minimize_step(C.byref(L), None, C.byref(sw), 0.3, None, 0, None) == _lib.HS_EINVAL
    assert lib.hs_relax_check(C.byref(L), None, 1, None, 0, None) == _lib.HS_EINVAL
    assert lib.hs_minimize_all(C.byref(L), None, C.byref(sw), 1, 0, None, 0, None) == _lib.HS_EINVAL
    buf = C.create_string_buffer(256)
    lib.hs_last_error(buf, 256)
    assert buf.value                                                            # a message was left


def _host_only_lattice(nx=64, ny=64):
    """An HsLattice whose checks pass on the host; its pointers are host buffers, so it may
    only reach code that refuses it before any launch."""
    import ctypes as C
    from hotspice_b200 import _lib
    keep = [C.create_string_buffer(16) for _ in range(5)]
    L = _lib.HsLattice()
    L.m, L.occ, L.mm, L.E_B, L.nonzero = (C.addressof(b) for b in keep)
    L.nx, L.ny, L.ux, L.uy, L.n_occ, L.beta_uniform = nx, ny, 1, 1, nx * ny, 1e20
    return L, keep


def test_metropolis_entry_points_validate_before_any_cuda_call():
    """hs_metropolis_step_noalloc checks the lattice, the plan and the Poisson radius before it
    sizes anything or touches the device: a NaN radius, an unknown sampling scheme and a
    Poisson grid beyond HS_POISSON_GRID_MAX are refused here, without a GPU."""
    import ctypes as C
    from hotspice_b200 import _lib
    lib = _lib.load()
    L, keep = _host_only_lattice()
    Cn, sw = _lib.HsCounters(), _lib.HsSwitchList()
    P = _lib.HsGridPlan()
    P.sample_scheme, P.r_cells, P.n_sc = _lib.HS_SAMPLE_POISSON, float('nan'), 1
    assert lib.hs_metropolis_step_noalloc(C.byref(L), C.byref(Cn), C.byref(sw), C.byref(P), None) == _lib.HS_EINVAL
    assert 'Poisson radius' in _lib.last_error()
    assert lib.hs_metropolis_scratch_bytes(C.byref(L), C.byref(P)) == -1
    P.sample_scheme = 7
    assert lib.hs_metropolis_step_noalloc(C.byref(L), C.byref(Cn), C.byref(sw), C.byref(P), None) == _lib.HS_EINVAL
    assert 'sample scheme' in _lib.last_error()
    # 40000^2 cells at radius 0: a background grid of ~3.2e9 cells (more than an int holds)
    Lb, keepb = _host_only_lattice(40000, 40000)
    P.sample_scheme, P.r_cells = _lib.HS_SAMPLE_POISSON, 0.0
    assert lib.hs_metropolis_step_noalloc(C.byref(Lb), C.byref(Cn), C.byref(sw), C.byref(P), None) == _lib.HS_ERANGE
    assert 'background grid' in _lib.last_error()
    assert lib.hs_metropolis_step(C.byref(Lb), C.byref(Cn), C.byref(sw), C.byref(P), None, 0, None) == _lib.HS_ERANGE


def test_progress_with_no_finite_limit_is_refused():
    """progress() with t_max and MCsteps_max both infinite would never end: the C ABI and the
    host-side check refuse it."""
    import ctypes as C
    import math
    from hotspice_b200 import _lib
    from hotspice_b200.core import check_progress_limits
    lib = _lib.load()
    Cn = _lib.HsCounters()
    assert lib.hs_progress_arm(C.byref(Cn), 4, math.inf, math.inf, None) == _lib.HS_EINVAL
    assert 'both infinite' in _lib.last_error()
    with pytest.raises(ValueError):
        check_progress_limits(math.inf, math.inf)
    check_progress_limits(math.inf, 4.0)
    check_progress_limits(1e-3, math.inf)
