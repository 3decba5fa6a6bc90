"""CPU tests of the reservoir I/O host logic (hotspice_b200/io.py): region bins of the output
readers and the field / progress stages the inputters hand to the device."""
import math
from types import SimpleNamespace

import numpy as np
import pytest


@pytest.mark.parametrize('n_bins,n_cells', [(4, 16), (3, 12), (8, 256), (5, 7), (7, 5), (1, 9)])
def test_region_bins_match_reference_formula(n_bins, n_cells):
    """hotspice/io.py:350-351: bin = int(linspace(0, n_bins (1 - 1e-15), n_cells)); each bin is a
    contiguous cell range [lo, hi) (possibly empty when there are more bins than cells)."""
    from hotspice_b200.io import _bins
    b, lo, hi = _bins(n_bins, n_cells)
    assert np.array_equal(b, np.linspace(0, n_bins * (1 - 1e-15), n_cells, dtype=int))
    for k in range(n_bins):
        assert np.array_equal(np.nonzero(b == k)[0], np.arange(lo[k], hi[k]))


def _mm(in_plane):
    return SimpleNamespace(in_plane=in_plane)


@pytest.mark.parametrize('half_period', [True, False])
@pytest.mark.parametrize('in_plane', [True, False])
def test_field_inputter_stages(half_period, in_plane):
    """hotspice/io.py:221-239 with sine=False: magnitude * value for t_max = 1 / f / (2 period) and
    n / (2 period) MC steps; a full period adds -magnitude * value for 0.5 / f and n / 2."""
    from hotspice_b200 import io as hio
    inp = hio.FieldInputter(hio.RandomScalarDatastream(), magnitude=2e-3, angle=7.0, n=3, frequency=50.0,
                            half_period=half_period)
    st = inp.stages(_mm(in_plane), 0.4)
    period = 1 / (1 + half_period)
    assert len(st) == (1 if half_period else 2)
    assert st[0].magnitude == 2e-3 * 0.4 and st[0].pattern is None
    assert st[0].angle == ((7.0 % math.tau) if in_plane else None)
    assert st[0].t_max == 1 / 50.0 / (2 * period) and st[0].mc_max == 3 / (2 * period)
    if not half_period:
        assert st[1].magnitude == -2e-3 * 0.4 and st[1].angle is None
        assert st[1].t_max == .5 / 50.0 and st[1].mc_max == 1.5
    assert inp.stages(_mm(in_plane), 1.0)[0].magnitude == 2e-3
    inp.sine = True
    assert inp.stages(_mm(in_plane), 0.4) is None          # host-stepped


def test_binary_and_perp_stages():
    from hotspice_b200 import io as hio
    b = hio.FieldInputterBinary(hio.RandomBinaryDatastream(), magnitudes=(.6, 1.5), frequency=2.0)
    assert [s.magnitude for s in b.stages(_mm(True), 0)] == [1.5 * (.6 / 1.5), -1.5 * (.6 / 1.5)]
    assert [s.magnitude for s in b.stages(_mm(True), 1)] == [1.5, -1.5]
    p = hio.PerpFieldInputter(hio.RandomBinaryDatastream(), magnitude=3e-3, angle=0.2, n=2, relax=False, frequency=4.0)
    mm = SimpleNamespace(in_plane=True, params=SimpleNamespace(UPDATE_SCHEME=__import__('hotspice_b200').Scheme.NEEL))
    st = p.stages(mm, 1)
    assert [s.magnitude for s in st] == [3e-3, -3e-3]
    assert all(s.angle == 0.2 + math.pi / 2 for s in st) and all(s.t_max == 0.125 and s.mc_max == 2 for s in st)
    assert hio.PerpFieldInputter(hio.RandomBinaryDatastream(), relax=True).stages(mm, 1) is None
    with pytest.raises(AttributeError):
        p.stages(SimpleNamespace(in_plane=False, params=mm.params), 1)


def test_steps_transform_piecewise_linear():
    """hotspice/io.py:483-500."""
    from hotspice_b200 import io as hio
    s = hio.OOPSquareChessStepsInputter(hio.RandomScalarDatastream(), magnitude=1.0, magnitude_range=0.2, transition_range=0.4)
    sw = 0.5 - 0.4 / 2
    for v in (0.0, 0.1, 0.29, 0.3, 0.5, 0.65, 0.7, 0.71, 0.95, 1.0):
        if v < sw:
            ref = -1.0 + v * 0.2 / sw
        elif v > 1 - sw:
            ref = 1.0 + (v - 1) * 0.2 / sw
        else:
            ref = 2 * (1.0 - 0.2) / 0.4 * (v - 0.5)
        assert s.transform(v) == ref
    b = hio.OOPSquareChessStepsInputter(hio.RandomBinaryDatastream(), magnitude=2.0)
    assert b.transform(0) == -2.0 and b.transform(1) == 2.0


def test_integer_datastream_bits():
    from hotspice_b200 import io as hio
    d = hio.RandomIntegerDatastream(num_bits=5)
    assert d.as_bits(6).tolist() == [0, 1, 1, 0, 0]
    assert d.as_bits(6, endianness='big').tolist() == [0, 0, 1, 1, 0]
    inp = hio.OOPSquareChessFieldInputter(d)
    assert hio._expand(inp, np.array([6, 1])).tolist() == [0, 1, 1, 0, 0, 1, 0, 0, 0, 0]
