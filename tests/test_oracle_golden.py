"""Pins the FP64 oracle against fixtures produced by the reference itself.

The reference run and the oracle consume identical Philox variates, so switch sequences,
counters, time and RNG call counts must agree exactly and energies to FP64 round-off."""
import numpy as np
import pytest

from cases import build_oracle, dipolar_like, load_fixture, load_specs, rel_err, run_io_oracle, run_relaxation
from oracle.philox import PhiloxStream, philox4x32_10, uniform53

SPECS = load_specs()


def test_philox_known_answers():
    """Random123 known-answer vectors for philox4x32-10."""
    cases = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
             ((0xffffffff,) * 4, (0xffffffff, 0xffffffff), (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
             ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
              (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]
    for ctr, key, want in cases:
        got = tuple(int(w) for w in philox4x32_10(*ctr, *key))
        assert got == want


def test_stream_transforms():
    s = PhiloxStream(123)
    u = uniform53(123, 0, 5)
    assert np.array_equal(s.random(5), u)
    assert s.call == 1
    assert s.randint(10) == int(np.floor(uniform53(123, 1, 1)[0] * 10))
    c = s.choice(7, 4)
    assert np.array_equal(c, np.floor(uniform53(123, 2, 4) * 7).astype(np.int64))
    e = s.exponential(scale=np.full((2, 3), 2.0), size=(2, 3))
    assert np.allclose(e, 2.0 * -np.log1p(-uniform53(123, 3, 6).reshape(2, 3)))
    assert np.all((u >= 0) & (u < 1))


@pytest.mark.parametrize('name', [n for n in SPECS if not SPECS[n].get('progress')])
def test_oracle_matches_reference(name):
    spec, fx = SPECS[name], load_fixture(name)
    mm = build_oracle(name, spec, fx)
    assert np.array_equal(mm.occupation, fx['occupation'])
    assert tuple(mm.unitcell) == tuple(fx['unitcell'])
    assert mm.PBC == bool(fx['PBC'])
    dip = dipolar_like(mm)
    if dip is not None:
        assert dip.kernels.shape == fx['kernels'].shape
        assert rel_err(dip.kernels, fx['kernels']) < 1e-13
        assert rel_err(dip.kernels_perpself, fx['kernels_perpself']) < 1e-13
        assert rel_err(dip.kernels_perpother, fx['kernels_perpother']) < 1e-13
        assert np.array_equal(dip.kernel_index, fx['kernel_index'])
        assert rel_err(dip.E, fx['E_dip_init']) < 1e-12
        assert rel_err(dip.E_perp, fx['E_dip_perp_init']) < 1e-12
    assert rel_err(mm.E, fx['E_init']) < 1e-12
    sw_y, sw_x, sw_step = [], [], []
    for s in range(spec.get('steps', 0)):
        idx = mm.update(**spec.get('update_kw', {}))
        if idx is not None:
            a = np.asarray(idx).reshape(2, -1)
            sw_y += a[0].tolist(); sw_x += a[1].tolist(); sw_step += [s] * a.shape[1]
        assert mm.rng.call == fx['calls'][s], f'RNG call count diverged at step {s}'
        assert mm.attempted_switches == fx['attempted'][s]
        assert mm.switches == fx['switches'][s]
        # t = tau * exp(b_min * beta) amplifies FP64 energy round-off by beta*|b| (~1e3)
        assert mm.t == pytest.approx(fx["t"][s], rel=1e-9, abs=0)
    assert np.array_equal(sw_y, fx['sw_y']) and np.array_equal(sw_x, fx['sw_x'])
    assert np.array_equal(sw_step, fx['sw_step'])
    run_relaxation(mm, spec)
    if spec.get('io') is not None:
        assert rel_err(run_io_oracle(mm, spec), fx['io_outputs']) < 1e-12
    if 'final_counts' in fx:
        assert [mm.switches, mm.attempted_switches, mm.rng.call] == fx['final_counts'].tolist()
    assert np.array_equal(mm.m, fx['m_final'])
    assert rel_err(mm.E, fx['E_final']) < 1e-11
    if dip is not None:
        assert rel_err(dip.E, fx['E_dip_final']) < 1e-11
        assert rel_err(dip.E_perp, fx['E_dip_perp_final']) < 1e-11


@pytest.mark.parametrize('name', [n for n in SPECS if SPECS[n].get('progress')])
def test_oracle_progress_matches_reference(name):
    spec, fx = SPECS[name], load_fixture(name)
    mm = build_oracle(name, spec, fx)
    dt, dmc = mm.progress(**spec['progress'])
    assert dt == pytest.approx(fx["progress"][0], rel=1e-9)
    assert dmc == pytest.approx(fx['progress'][1], rel=1e-12)
    assert mm.rng.call == int(fx['progress_calls'])
    assert np.array_equal(mm.m, fx['m_final'])
    assert rel_err(mm.E, fx['E_final']) < 1e-11


def test_hexagon_known_answer():
    """The reference's own known-answer test (tests/test_hexagon.py): every magnet of a
    kagome hexagon in a vortex state has E = -1e-7 m^2/a^3 (29 + 20 sqrt(3)/9)."""
    from oracle.geometry import ip_kagome
    from oracle.hotspice_oracle import OracleDipolar, OracleMagnets
    z = load_fixture('hexagon_kat')
    E_th = float(z['E_theory'])
    l, mom = 470e-9, 1.1278401e-15
    a = l / np.tan(30 * np.pi / 180)
    for nx in range(5, 11):
        for ny in range(3, 11):
            g = ip_kagome(a, nx, ny)
            m_ref, occ_ref, E_ref = (z[f'{nx}x{ny}_{i}'] for i in range(3))
            g.occupation = occ_ref.astype(int)
            dd = OracleDipolar()
            mm = OracleMagnets(g, m_ref, T=300, moment=mom, energies=[dd], m_perp_factor=0)
            assert np.allclose(dd.E[m_ref.astype(bool)], E_th)
            assert rel_err(dd.E, E_ref) < 1e-12


def test_poisson_reference_is_degenerate():
    """The reference's _select_Poisson passes metres into a cell-unit routine
    (hotspice/core.py:564 -> hotspice/poisson.py:77,99) and so always returns magnet (0,0);
    the oracle's compatibility mode reproduces the recorded selections."""
    from oracle.geometry import oop_square
    from oracle.hotspice_oracle import OracleDipolar, OracleMagnets
    sel = load_fixture('poisson_reference')['selections']
    mm = OracleMagnets(oop_square(200e-9, 16), np.ones((16, 16)), T=300, moment=1e-15, energies=[OracleDipolar()],
                       params=dict(UPDATE_SCHEME='Metropolis', MULTISAMPLING_SCHEME='Poisson'), seed=5,
                       poisson_compat=True)
    for s in sel:
        assert np.array_equal(mm.select(r=mm.calc_r(0.05)), s)


@pytest.mark.parametrize('w,h,r', [(48, 48, 6.0), (64, 40, 3.5), (30, 30, 9.0)])
def test_poisson_disc_cells_keeps_its_distance(w, h, r):
    """Cell-unit dart throwing (hotspice/poisson.py:72-128): every pair of accepted points is
    farther apart than r + 1 under the periodic metric, and the background grid is covered
    (no empty 2(r+1) x 2(r+1) window at the far side of the range)."""
    from oracle.hotspice_oracle import poisson_disc_cells
    for seed in range(3):
        s = PhiloxStream(100 + seed)
        pts = np.asarray(poisson_disc_cells(w, h, r, 4, s.random), dtype=float)
        assert len(pts) >= max(1, int(0.3 * w * h / (np.pi * (r + 1) ** 2)))
        d = np.abs(pts[:, None, :] - pts[None, :, :])
        d = np.minimum(d, np.array([w, h]) - d)
        d2 = (d ** 2).sum(-1) + np.eye(len(pts)) * 1e9
        assert d2.min() > (r + 1) ** 2


def test_square_vertex_fractions_match_reference():
    """The oracle's vertex counting equals the reference's count_square_vertices
    (examples/IP_SquareVertices.py:19-35, run unmodified by make_golden.py)."""
    from oracle.hotspice_oracle import square_vertex_fractions
    z = load_fixture('square_vertices')
    for k in range(int(z['n_cases'])):
        assert np.allclose(square_vertex_fractions(z[f'm_{k}']), z[f'fractions_{k}'], rtol=0, atol=1e-15), k
