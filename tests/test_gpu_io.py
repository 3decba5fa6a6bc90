"""Reservoir inputs and outputs (hotspice/io.py) on the device against the reference fixtures.

* run_sequence (device field writes, device-armed progress() in persistent engine launches,
  device readouts, one synchronisation) reproduces the reference run: readouts, final spins,
  switch / attempt / Philox-call counts. Readouts are sums of spins times FP64 weights in a
  different order than numpy's: max|dr| / max|r| <= 1e-12.
* The per-value public API (Inputter.input + OutputReader.read_state) equals run_sequence.
* set_field_device equals the host set_field to FP64 rounding.
"""
import numpy as np
import pytest
import torch

from cases import load_fixture, load_specs, product_io_objects, rel_err
from gpu_cases import build_product

pytestmark = pytest.mark.gpu
SPECS = load_specs()
IO = [n for n in SPECS if SPECS[n].get('io') is not None]


def _np(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize('name', IO)
def test_sequence_matches_reference(name):
    from hotspice_b200 import io as hio
    spec, fx = SPECS[name], load_fixture(name)
    mp = build_product(name)
    inp, rd = product_io_objects(mp, spec['io'])
    values, out = hio.run_sequence(mp, inp, spec['io']['values'], rd)
    assert rel_err(_np(out), fx['io_outputs']) < 1e-12
    c = mp._read_counters()
    assert [int(c['switches']), int(c['attempted']), int(c['rng_call'])] == fx['final_counts'].tolist()
    assert np.array_equal(_np(mp.m), fx['m_final'])
    assert rel_err(_np(mp.E), fx['E_final']) < 2e-6


@pytest.mark.parametrize('name', IO)
def test_public_api_equals_sequence(name):
    from hotspice_b200 import io as hio
    spec = SPECS[name]
    a, b = build_product(name), build_product(name)
    inp_a, rd_a = product_io_objects(a, spec['io'])
    inp_b, rd_b = product_io_objects(b, spec['io'])
    _, out = hio.run_sequence(a, inp_a, spec['io']['values'], rd_a)
    rows = []
    for v in spec['io']['values']:
        inp_b.input(b, values=[v])
        rows.append(rd_b.read_state(b).clone())
    assert torch.equal(out, torch.stack(rows))
    assert torch.equal(a._m_dev, b._m_dev)
    assert a._read_counters()['rng_call'] == b._read_counters()['rng_call']


@pytest.mark.parametrize('in_plane', [False, True])
def test_set_field_device_equals_host(in_plane):
    import hotspice_b200 as hs
    if in_plane:
        mm = hs.ASI.IP_Kagome(500e-9, 24, energies=[hs.ZeemanEnergy(1e-3, 0.4)])
        mm.moment = np.linspace(1e-15, 2e-15, mm.nx * mm.ny).reshape(mm.ny, mm.nx)
    else:
        mm = hs.ASI.OOP_Square(200e-9, 24, energies=[hs.ZeemanEnergy(1e-3)])
    Z = mm.get_energy('Zeeman')
    pat = torch.as_tensor(((mm.ixx + mm.iyy) % 3 - 1).astype(np.float32), device=mm.device)
    Z.set_field_device(2.5e-3, pattern=pat, angle=0.7 if in_plane else None)
    dev = (_np(Z.E_factor).copy(), _np(Z.E_factor_perp).copy(), _np(Z._ef32).copy())
    Z.set_field(magnitude=2.5e-3 * _np(pat).astype(float), angle=0.7 if in_plane else None)
    host = (_np(Z.E_factor), _np(Z.E_factor_perp), _np(Z._ef32))
    assert rel_err(dev[0], host[0]) < 1e-15
    if in_plane:
        assert rel_err(dev[1], host[1]) < 1e-15
    assert rel_err(dev[2], host[2]) < 1e-7
    assert np.array_equal(np.asarray(Z.magnitude), 2.5e-3 * _np(pat).astype(float))


def test_large_reservoir_sequence():
    """A 256^2 OOP_Square reservoir driven by 40 checkerboard inputs: readouts in [-1, 1], the
    device-armed progress advances at most MCsteps_max per input, and the run is the same as
    the per-value API."""
    import hotspice_b200 as hs
    from hotspice_b200 import io as hio
    def make():
        return hs.ASI.OOP_Square(200e-9, 256, T=300, E_B=5e-20, moment=1.1e-15, pattern='random', seed=4,
                                 energies=[hs.DipolarEnergy(cutoff_range=8.3 * 200e-9), hs.ZeemanEnergy(0)])
    vals = (np.arange(40) * 7 % 5 > 1).astype(int)
    a = make()
    inp = hio.OOPSquareChessFieldInputter(hio.RandomBinaryDatastream(), magnitude=8e-4, n=0.05, frequency=1e3)
    rd = hio.OOPSquareChessOutputReader(8, 8, a)
    att0 = a.attempted_switches
    _, out = hio.run_sequence(a, inp, vals, rd)
    o = _np(out)
    assert o.shape == (40, 64) and np.all(np.abs(o) <= 1 + 1e-12)
    assert (a.attempted_switches - att0) / a.n <= 40 * 0.05 + 40 / a.n + 1e-9
    b = make()
    rows = []
    for v in vals:
        inp.input(b, values=[v])
        rows.append(rd.read_state(b).clone())
    assert torch.equal(out, torch.stack(rows))


@pytest.mark.parametrize('name', ['io_chess_oop16', 'io_steps_oop12_metro', 'io_field_pin16', 'io_perp_pin12_progress'])
def test_batch_equals_sequences(name):
    """run_batch (one engine launch per input stage for all instances) gives every instance
    the result of its own run_sequence, bit for bit: different seeds and input values per
    instance."""
    from hotspice_b200 import io as hio
    spec = SPECS[name]
    base = np.asarray(spec['io']['values'])
    vals = np.stack([base, base[::-1], np.roll(base, 1)])
    seeds = [spec['seed'], spec['seed'] + 100, spec['seed'] + 200]
    alone = []
    for v, sd in zip(vals, seeds):
        mm = build_product(name, seed=sd)
        inp, rd = product_io_objects(mm, spec['io'])
        _, out = hio.run_sequence(mm, inp, v, rd)
        alone.append((out, mm._m_dev.clone(), mm._read_counters()))
    mms = [build_product(name, seed=sd) for sd in seeds]
    objs = [product_io_objects(mm, spec['io']) for mm in mms]
    outs = hio.run_batch(mms, objs[0][0], vals, [o[1] for o in objs])
    for i, mm in enumerate(mms):
        assert torch.equal(outs[i], alone[i][0]), f'instance {i}: readouts differ'
        assert torch.equal(mm._m_dev, alone[i][1])
        c = mm._read_counters()
        for k in ('switches', 'attempted', 'rng_call', 't'):
            assert c[k] == alone[i][2][k], (i, k)


def test_batch_refuses_host_inputs():
    import hotspice_b200 as hs
    from hotspice_b200 import io as hio
    mm = hs.ASI.IP_Pinwheel(300e-9, 12, energies=[hs.DipolarEnergy(), hs.ZeemanEnergy(0)])
    with pytest.raises(NotImplementedError):
        hio.run_batch([mm], hio.PerpFieldInputter(hio.RandomBinaryDatastream(), relax=True), [0, 1])
