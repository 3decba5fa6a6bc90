"""Generate golden fixtures by running the reference Hotspice NumPy path.

Usage (only where the reference source tree is present):
    python tests/golden/make_golden.py --ref <reference checkout>   (or HOTSPICE_REFERENCE=<dir>)
    python tests/golden/make_golden.py --ref <dir> --vertices        (only square_vertices.npz)

The reference package is imported unmodified: ``hotspice/__init__.py`` (which pulls in the
GUI and plotting modules) is bypassed by registering a bare package module, and the three
display-only imports of ``hotspice/utils.py`` (colorama, IPython, matplotlib.figure) are
satisfied by inert stubs. Every random draw the hot path makes (``mm.rng`` and the global
``numpy.random.{randint,choice,random}``; hotspice/core.py:83,493,527-538,598-600,666-692)
is routed through ``oracle.philox.PhiloxStream`` so the oracle and the CUDA kernels can
consume the identical variates.

Each scenario writes ``tests/golden/<name>.npz`` with the inputs, the per-step switch
records and the energies the reference produced. The fixtures are small (lattices of at
most 32x32, at most a few hundred steps).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle.philox import PhiloxStream  # noqa: E402


def load_reference(ref_root):
    colorama = types.ModuleType('colorama')
    colorama.init = lambda *a, **k: None

    class _Blank:
        def __getattr__(self, name):
            return ''
    colorama.Fore = colorama.Style = _Blank()
    ipy = types.ModuleType('IPython')
    ipy_t = types.ModuleType('IPython.terminal')
    ipy_e = types.ModuleType('IPython.terminal.embed')
    ipy_e.InteractiveShellEmbed = object
    mpl = types.ModuleType('matplotlib')
    mpl_f = types.ModuleType('matplotlib.figure')
    mpl_f.Figure = object
    for name, mod in (('colorama', colorama), ('IPython', ipy), ('IPython.terminal', ipy_t),
                      ('IPython.terminal.embed', ipy_e), ('matplotlib', mpl), ('matplotlib.figure', mpl_f)):
        sys.modules.setdefault(name, mod)
    os.environ['HOTSPICE_USE_GPU'] = 'False'
    pkg = types.ModuleType('hotspice')
    pkg.__path__ = [os.path.join(ref_root, 'hotspice')]
    sys.modules['hotspice'] = pkg
    import hotspice.config  # noqa: F401
    import hotspice.utils  # noqa: F401
    import hotspice.energies  # noqa: F401
    import hotspice.poisson  # noqa: F401
    import hotspice.core  # noqa: F401
    import hotspice.ASI  # noqa: F401
    # hotspice/io.py imports show_m from the plotting module: an inert stand-in
    pt = types.ModuleType('hotspice.plottools')
    pt.show_m = lambda *a, **k: None
    sys.modules['hotspice.plottools'] = pt
    import hotspice.io  # noqa: F401
    return sys.modules['hotspice']


def route_rng(mm, stream):
    """Replace every random source of the hot path with ``stream``."""
    mm.rng = stream
    np.random.randint = stream.randint
    np.random.choice = stream.choice
    np.random.random = stream.random
    np.random.permutation = stream.permutation


def lognormal_EB(mean, sigma, shape, seed):
    g = np.random.Generator(np.random.PCG64(seed))
    return mean * g.lognormal(-sigma ** 2 / 2, sigma, size=shape)


def random_pm1(shape, seed):
    g = np.random.Generator(np.random.PCG64(seed))
    return g.integers(0, 2, size=shape) * 2 - 1


SCENARIOS = []


def scenario(fn):
    SCENARIOS.append(fn)
    return fn


def _lattice(hs, spec):
    kind = spec['lattice']
    kw = dict(spec.get('kw', {}))
    if kind == 'OOP_Square':
        return hs.ASI.OOP_Square(spec['a'], nx=spec['nx'], ny=spec['ny'], **kw)
    if kind == 'IP_Pinwheel':
        return hs.ASI.IP_Pinwheel(spec['a'], nx=spec['nx'], ny=spec['ny'], **kw)
    if kind == 'IP_Square':
        return hs.ASI.IP_Square(spec['a'], nx=spec['nx'], ny=spec['ny'], **kw)
    if kind == 'IP_Kagome':
        return hs.ASI.IP_Kagome(spec['a'], nx=spec['nx'], ny=spec['ny'], **kw)
    raise ValueError(kind)


def io_objects(hs, io, mm):
    """The reference Inputter / OutputReader of an 'io' scenario (hotspice/io.py)."""
    hio = sys.modules['hotspice.io']
    p = io['params']
    kind = io['inputter']
    if kind == 'field':
        inp = hio.FieldInputter(hio.RandomScalarDatastream(), magnitude=p['magnitude'], angle=p['angle'], n=p['n'],
                                sine=p.get('sine', False), frequency=p['frequency'], half_period=p['half_period'])
    elif kind == 'perp':
        inp = hio.PerpFieldInputter(hio.RandomBinaryDatastream(), magnitude=p['magnitude'], angle=p['angle'], n=p['n'],
                                    relax=p['relax'], frequency=p['frequency'])
    elif kind == 'chess':
        inp = hio.OOPSquareChessFieldInputter(hio.RandomBinaryDatastream(), magnitude=p['magnitude'], n=p['n'],
                                              frequency=p['frequency'])
    elif kind == 'steps':
        ds = hio.RandomBinaryDatastream() if p.get('binary') else hio.RandomScalarDatastream()
        inp = hio.OOPSquareChessStepsInputter(ds, magnitude=p['magnitude'], magnitude_range=p['magnitude_range'],
                                              transition_range=p['transition_range'], n=p['n'], frequency=p['frequency'])
    else:
        raise ValueError(kind)
    rp = io['reader_params']
    rd = {'full': lambda: hio.FullOutputReader(mm), 'regional': lambda: hio.RegionalOutputReader(rp['nx'], rp['ny'], mm),
          'chess': lambda: hio.OOPSquareChessOutputReader(rp['nx'], rp['ny'], mm)}[io['reader']]()
    return inp, rd


def run_spec(hs, spec):
    """Build the reference Magnets for ``spec``, run it, and collect the record."""
    E = hs.energies
    energies = []
    for e in spec['energies']:
        if e['type'] == 'dipolar':
            energies.append(E.DipolarEnergy(cutoff_range=e.get('cutoff', np.inf)))
        elif e['type'] == 'dimonopolar':
            energies.append(E.DiMonopolarEnergy(prefactor=e.get('prefactor', 1.0), d=e['d'], small_d=e['small_d']))
        elif e['type'] == 'zeeman':
            energies.append(E.ZeemanEnergy(magnitude=e['B'], angle=e.get('angle', 0.0)))
        elif e['type'] == 'exchange':
            energies.append(E.ExchangeEnergy(J=e['J']))
    ny, nx = spec['ny'], spec['nx']
    m0 = random_pm1((ny, nx), spec['seed'])
    EB = spec['E_B']
    if isinstance(EB, dict):
        EB = lognormal_EB(EB['mean'], EB['sigma'], (ny, nx), spec['seed'] + 1)
    params = hs.core.SimParams(**spec.get('params', {}))
    kw = dict(spec.get('kw', {}))
    mm = _lattice(hs, dict(spec, kw=dict(kw, T=spec['T'], E_B=EB, moment=spec['moment'], pattern='uniform',
                                         energies=energies, params=params)))
    # an ndarray pattern cannot be passed to the constructor (hotspice/core.py:104,172 read
    # self.shape before self.m exists), so set the start state afterwards
    mm.initialize_m(m0)
    stream = PhiloxStream(spec['seed'])
    route_rng(mm, stream)
    rec = dict(m0=m0, E_B=np.asarray(EB, dtype=float) * np.ones((ny, nx)), occupation=mm.occupation,
               unitcell=np.array([mm.unitcell.x, mm.unitcell.y]), PBC=np.array(mm.PBC))
    dip = mm.get_energy('dipolar', verbose=False) or mm.get_energy('dimonopolar', verbose=False)
    if dip is not None:
        rec['kernels'] = dip.kernel_unitcell
        rec['kernels_perpself'] = dip.kernel_perpself_unitcell
        rec['kernels_perpother'] = dip.kernel_perpother_unitcell
        rec['kernel_index'] = dip.kernel_unitcell_indices
        rec['E_dip_init'] = dip.E.copy()
        rec['E_dip_perp_init'] = dip.E_perp.copy()
    rec['E_init'] = mm.E.copy()
    steps = spec.get('steps', 0)
    sw_y, sw_x, sw_step, t_hist, att_hist, swc_hist, call_hist = [], [], [], [], [], [], []
    kwargs = spec.get('update_kw', {})
    for s in range(steps):
        idx = mm.update(**kwargs)
        if idx is not None:
            arr = np.asarray(idx).reshape(2, -1)
            sw_y.extend(arr[0].tolist()); sw_x.extend(arr[1].tolist()); sw_step.extend([s] * arr.shape[1])
        t_hist.append(mm.t); att_hist.append(mm.attempted_switches); swc_hist.append(mm.switches)
        call_hist.append(stream.call)
    rec.update(sw_y=np.array(sw_y, dtype=np.int64), sw_x=np.array(sw_x, dtype=np.int64),
               sw_step=np.array(sw_step, dtype=np.int64), t=np.array(t_hist), attempted=np.array(att_hist),
               switches=np.array(swc_hist), calls=np.array(call_hist, dtype=np.int64))
    if spec.get('progress'):
        t0 = mm.t
        dt, dmc = mm.progress(**spec['progress'])
        rec['progress'] = np.array([dt, dmc])
        rec['progress_calls'] = np.array(stream.call)
    if spec.get('relax') is not None:
        mm.relax(**spec['relax'])
    if spec.get('minimize') is not None:
        mm.minimize(**spec['minimize'])
    if spec.get('io') is not None:
        inp, rd = io_objects(hs, spec['io'], mm)
        outs = []
        for v in spec['io']['values']:
            inp.input(mm, values=[v])
            outs.append(np.asarray(rd.read_state(mm), dtype=float).copy())
        rec['io_outputs'] = np.array(outs)
    rec['final_counts'] = np.array([mm.switches, mm.attempted_switches, stream.call], dtype=np.int64)
    rec['m_final'] = mm.m.copy()
    rec['E_final'] = mm.E.copy()
    if dip is not None:
        rec['E_dip_final'] = dip.E.copy()
        rec['E_dip_perp_final'] = dip.E_perp.copy()
    return rec


BASE_OOP = dict(lattice='OOP_Square', a=200e-9, moment=1.1e-15, T=300.0, E_B=5e-20)
BASE_PIN = dict(lattice='IP_Pinwheel', a=300e-9, moment=1e-15, T=300.0, E_B=dict(mean=6e-20, sigma=0.05))

SPECS = {
    # config-1 shape at reduced size: full kernel, Néel
    'neel_oop16': dict(BASE_OOP, nx=16, ny=16, seed=11, energies=[dict(type='dipolar')], steps=300),
    'neel_oop12x9_pbc': dict(BASE_OOP, nx=12, ny=9, seed=12, kw=dict(PBC=True), energies=[dict(type='dipolar')], steps=200),
    'neel_oop16_parabolic': dict(BASE_OOP, nx=16, ny=16, seed=13, energies=[dict(type='dipolar'), dict(type='zeeman', B=2e-3)],
                                 params=dict(ENERGY_BARRIER_METHOD='parabolic'), steps=150),
    'neel_oop16_Tfield': dict(BASE_OOP, nx=16, ny=16, seed=14, T='field', energies=[dict(type='dipolar')], steps=150),
    # two-channel Néel with E_perp (in-plane)
    'neel_pin16_perp': dict(BASE_PIN, nx=16, ny=16, seed=21,
                            energies=[dict(type='dipolar'), dict(type='zeeman', B=1e-3, angle=math.radians(22.5))], steps=200),
    'neel_kagome_perp': dict(BASE_PIN, lattice='IP_Kagome', a=1e-6, nx=20, ny=15, seed=22,
                             energies=[dict(type='dipolar', cutoff=2.2e-6)], steps=120),
    # config-2 shape at reduced size: cutoff + Zeeman, Metropolis grid
    'metro_pin32_grid': dict(BASE_PIN, nx=32, ny=32, seed=31,
                             energies=[dict(type='dipolar', cutoff=5 * 300e-9), dict(type='zeeman', B=1e-3, angle=math.radians(22.5))],
                             steps=120, update_kw=dict(r=4 * 300e-9)),
    'metro_pin24_pbc': dict(BASE_PIN, nx=24, ny=24, seed=32, kw=dict(PBC=True),
                            energies=[dict(type='dipolar', cutoff=4 * 300e-9)], steps=100, update_kw=dict(r=3 * 300e-9)),
    # more than 20 switches per sublattice -> truncated 41x41 convolution branch
    'metro_oop32_trunc_pbc': dict(BASE_OOP, nx=32, ny=32, seed=33, kw=dict(PBC=True), T=2000.0, moment=2e-16,
                                  energies=[dict(type='dipolar')], steps=60, update_kw=dict(r=200e-9)),
    'metro_oop30_trunc': dict(BASE_OOP, nx=30, ny=26, seed=34, T=2000.0, moment=2e-16,
                              energies=[dict(type='dipolar')], steps=60, update_kw=dict(r=200e-9)),
    'metro_oop16_time': dict(BASE_OOP, nx=16, ny=16, seed=35, energies=[dict(type='dipolar')], steps=60,
                             params=dict(METROPOLIS_TIME=True), update_kw=dict(r=600e-9)),
    'metro_kagome_grid': dict(BASE_PIN, lattice='IP_Kagome', a=1e-6, nx=24, ny=19, seed=36,
                              energies=[dict(type='dipolar', cutoff=2e-6), dict(type='zeeman', B=2e-3, angle=0.3)],
                              steps=80, update_kw=dict(r=1.5e-6)),
    'metro_oop16_single': dict(BASE_OOP, nx=16, ny=16, seed=37, energies=[dict(type='dipolar')], steps=100,
                               params=dict(MULTISAMPLING_SCHEME='single')),
    # exchange-only Ising under Wolff near T_c = 2.269 J / kB
    'wolff_oop32_pbc': dict(BASE_OOP, nx=32, ny=32, seed=41, kw=dict(PBC=True), T=2.269e-21 / 1.380649e-23,
                            moment=1e-15, E_B=0.0, energies=[dict(type='exchange', J=1e-21)], steps=40,
                            params=dict(UPDATE_SCHEME='Wolff', MULTISAMPLING_SCHEME='cluster')),
    'wolff_oop20_open': dict(BASE_OOP, nx=20, ny=18, seed=42, T=150.0, moment=1e-15, E_B=0.0,
                             energies=[dict(type='exchange', J=1e-21)], steps=30,
                             params=dict(UPDATE_SCHEME='Wolff', MULTISAMPLING_SCHEME='cluster')),
    # exchange + dipolar under Néel (exchange recompute per switch)
    'neel_oop16_exchange': dict(BASE_OOP, nx=16, ny=16, seed=43, energies=[dict(type='dipolar'), dict(type='exchange', J=3e-21)],
                                steps=100),
    # progress() loop semantics (t_max / MCsteps_max stopping rule)
    'progress_oop12': dict(BASE_OOP, nx=12, ny=12, seed=51, energies=[dict(type='dipolar')], steps=0,
                           progress=dict(t_max=1e-3, MCsteps_max=0.5)),
    'progress_pin16_metro': dict(BASE_PIN, nx=16, ny=16, seed=52, energies=[dict(type='dipolar', cutoff=1.2e-6)], steps=0,
                                 params=dict(UPDATE_SCHEME='Metropolis'), progress=dict(t_max=1.0, MCsteps_max=3.0, r=900e-9)),
    # DiMonopolarEnergy (two opposite charges per magnet): two-channel Néel with E_perp
    'neel_pin16_dimono': dict(BASE_PIN, nx=16, ny=16, seed=61,
                              energies=[dict(type='dimonopolar', d=120e-9, small_d=60e-9),
                                        dict(type='zeeman', B=1e-3, angle=math.radians(22.5))], steps=150),
    'neel_kagome_dimono': dict(BASE_PIN, lattice='IP_Kagome', a=1e-6, nx=12, ny=11, seed=62,
                               energies=[dict(type='dimonopolar', prefactor=0.7, d=400e-9, small_d=150e-9)], steps=100),
    # multi-switch updates (E_perp keeps its sign there) and METROPOLIS_TIME barriers from E_perp
    'metro_sq16_dimono_pbc': dict(BASE_PIN, lattice='IP_Square', a=400e-9, nx=16, ny=16, seed=63, kw=dict(PBC=True),
                                  T=1500.0, energies=[dict(type='dimonopolar', d=150e-9, small_d=70e-9)], steps=60,
                                  params=dict(METROPOLIS_TIME=True), update_kw=dict(r=600e-9)),
    # relax() / _minimize_all() (sub-grid sweeps) and minimize() (sequential), from random states
    'relax_oop24': dict(BASE_OOP, nx=24, ny=24, seed=71, energies=[dict(type='dipolar')], steps=0, relax={}),
    'relax_pin20_pbc_barrier': dict(BASE_PIN, nx=20, ny=20, seed=72, kw=dict(PBC=True), E_B=3e-20,
                                    energies=[dict(type='dipolar', cutoff=6 * 300e-9), dict(type='zeeman', B=2e-3, angle=0.4)],
                                    steps=0, relax=dict(ignore_barrier=False)),
    'relax_kagome_exchange': dict(BASE_PIN, lattice='IP_Kagome', a=1e-6, nx=20, ny=17, seed=73,
                                  energies=[dict(type='dipolar', cutoff=3e-6), dict(type='exchange', J=2e-20)],
                                  steps=0, relax={}),
    'relax_oop16_simultaneous': dict(BASE_OOP, nx=16, ny=16, seed=74, energies=[dict(type='dipolar'), dict(type='zeeman', B=5e-4)],
                                     steps=0, relax=dict(_simultaneous=True)),
    'relax_sq16_dimono': dict(BASE_PIN, lattice='IP_Square', a=400e-9, nx=16, ny=16, seed=75,
                              energies=[dict(type='dimonopolar', d=150e-9, small_d=70e-9)], steps=0, relax={}),
    'minimize_oop16': dict(BASE_OOP, nx=16, ny=16, seed=76, energies=[dict(type='dipolar'), dict(type='zeeman', B=3e-4)],
                           steps=0, minimize={}),
    'minimize_pin16': dict(BASE_PIN, nx=16, ny=16, seed=77, energies=[dict(type='dipolar')], steps=0, minimize={}),
    # reservoir inputs and outputs (hotspice/io.py): field stimuli + progress()/minimize(), readouts
    'io_chess_oop16': dict(BASE_OOP, nx=16, ny=16, seed=81, energies=[dict(type='dipolar'), dict(type='zeeman', B=0.0)], steps=0,
                           io=dict(inputter='chess', params=dict(magnitude=4e-4, n=2, frequency=1.0), reader='chess',
                                   reader_params=dict(nx=4, ny=4), values=[1, 0, 0, 1, 1, 0])),
    'io_steps_oop12_metro': dict(BASE_OOP, nx=12, ny=12, seed=82, energies=[dict(type='dipolar'), dict(type='zeeman', B=0.0)],
                                 steps=0, params=dict(UPDATE_SCHEME='Metropolis'),
                                 io=dict(inputter='steps', params=dict(magnitude=6e-4, magnitude_range=2e-4, transition_range=0.4,
                                                                       n=1.0, frequency=1.0),
                                         reader='chess', reader_params=dict(nx=2, ny=3), values=[0.1, 0.45, 0.62, 0.95, 0.3])),
    'io_field_pin16': dict(BASE_PIN, nx=16, ny=16, seed=83, energies=[dict(type='dipolar', cutoff=1.5e-6), dict(type='zeeman', B=0.0)],
                           steps=0, io=dict(inputter='field', params=dict(magnitude=4e-3, angle=0.3, n=1.0, frequency=1.0,
                                                                         half_period=True),
                                            reader='regional', reader_params=dict(nx=4, ny=2), values=[0.3, -0.8, 0.1, 0.9, -0.55])),
    'io_sine_oop12': dict(BASE_OOP, nx=12, ny=12, seed=86, energies=[dict(type='dipolar'), dict(type='zeeman', B=0.0)], steps=0,
                          io=dict(inputter='field', params=dict(magnitude=1.5e-3, angle=0.0, n=0.5, frequency=2e3, half_period=True,
                                                                sine=True),
                                  reader='chess', reader_params=dict(nx=2, ny=2), values=[1.0, -0.6, 0.8])),
    'io_perp_pin12_relax': dict(BASE_PIN, nx=12, ny=12, seed=84, energies=[dict(type='dipolar'), dict(type='zeeman', B=0.0)], steps=0,
                                io=dict(inputter='perp', params=dict(magnitude=3e-3, angle=0.2, n=2, relax=True, frequency=1.0),
                                        reader='full', reader_params={}, values=[0, 1, 1, 0])),
    'io_perp_pin12_progress': dict(BASE_PIN, nx=12, ny=12, seed=85, energies=[dict(type='dipolar'), dict(type='zeeman', B=0.0)],
                                   steps=0, io=dict(inputter='perp', params=dict(magnitude=2e-3, angle=0.2, n=2, relax=False,
                                                                                 frequency=1.0),
                                                    reader='regional', reader_params=dict(nx=3, ny=3), values=[1, 0, 1])),
}
for name in ('metro_sq16_dimono_pbc', 'metro_pin32_grid', 'metro_pin24_pbc', 'metro_oop32_trunc_pbc', 'metro_oop30_trunc',
             'metro_oop16_time', 'metro_kagome_grid', 'metro_oop16_single'):
    SPECS[name].setdefault('params', {})['UPDATE_SCHEME'] = 'Metropolis'


def make_T_field(spec):
    ny, nx = spec['ny'], spec['nx']
    yy, xx = np.mgrid[0:ny, 0:nx]
    return 280.0 + 40.0 * (xx / max(nx - 1, 1)) + 5.0 * (yy % 3)


def hexagon_kat(hs):
    """tests/test_hexagon.py of the reference: a trimmed kagome hexagon in a vortex state."""
    out = {}
    l = 470e-9
    mom = 1.1278401e-15
    a = l / np.tan(30 * np.pi / 180)
    for nx in range(5, 11):
        for ny in range(3, 11):
            mm = hs.ASI.IP_Kagome(a, nx=nx, ny=ny, moment=mom, energies=[dd := hs.energies.DipolarEnergy()],
                                  T=300, m_perp_factor=0, PBC=False)
            mm.occupation[3:, :] = mm.m[3:, :] = 0
            mm.occupation[:, 5:] = mm.m[:, 5:] = 0
            mm.m[(0, 0, 1), (1, 3, 4)] *= -1
            mm.update_energy()
            out[f'{nx}x{ny}'] = (mm.m.copy(), mm.occupation.copy(), dd.E.copy())
    return out, -1e-7 * mom * mom / a ** 3 * (29 + 20 * np.sqrt(3) / 9)


def reference_vertex_counter(ref_root):
    """The reference's count_square_vertices (examples/IP_SquareVertices.py:19-35), taken from
    the example file as written and executed unmodified (the example module itself imports
    plotting packages, so only this function's source is compiled)."""
    import ast
    from scipy import signal
    path = os.path.join(ref_root, 'examples', 'IP_SquareVertices.py')
    src = open(path).read()
    fn = next(n for n in ast.parse(src).body if isinstance(n, ast.FunctionDef) and n.name == 'count_square_vertices')
    fn.returns = None
    for a in fn.args.args:
        a.annotation = None
    mod = ast.Module(body=[fn], type_ignores=[])
    env = {'np': np, 'signal': signal}
    exec(compile(mod, path, 'exec'), env)
    return env['count_square_vertices']


def square_vertices(hs, ref_root):
    """Vertex fractions of IP_Square states (random, ground state, and lightly annealed ones)
    by the reference's own counting function."""
    count = reference_vertex_counter(ref_root)
    out = {}
    cases = [(12, True, 'random', 1), (20, True, 'random', 2), (16, True, 'afm', 3), (18, False, 'random', 4),
             (24, True, 'biased', 5)]
    for k, (n, pbc, pattern, seed) in enumerate(cases):
        mm = hs.ASI.IP_Square(1e-6, n, PBC=pbc, moment=3e-17, T=300, energies=[hs.energies.ZeemanEnergy()])
        g = np.random.Generator(np.random.PCG64(seed))
        if pattern == 'random':
            mm.m = mm.occupation * (g.integers(0, 2, size=mm.m.shape) * 2 - 1)
        elif pattern == 'biased':
            mm.m = mm.occupation * np.where(g.random(mm.m.shape) < 0.8, 1, -1)
        else:
            mm.initialize_m('afm')
        out[f'm_{k}'] = np.asarray(mm.m, dtype=np.int8)
        out[f'pbc_{k}'] = np.asarray(pbc)
        out[f'fractions_{k}'] = np.asarray(count(mm), dtype=float)
    out['n_cases'] = np.asarray(len(cases))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--ref', default=os.environ.get('HOTSPICE_REFERENCE'),
                    help='reference checkout (or set HOTSPICE_REFERENCE)')
    ap.add_argument('--only', default=None, help='comma-separated scenario names; merged into specs.json')
    ap.add_argument('--vertices', action='store_true', help='write only square_vertices.npz')
    args = ap.parse_args()
    if not args.ref:
        ap.error('the reference checkout is required: --ref <dir> or HOTSPICE_REFERENCE=<dir>')
    hs = load_reference(args.ref)
    if args.vertices:
        np.savez_compressed(os.path.join(HERE, 'square_vertices.npz'), **square_vertices(hs, args.ref))
        return
    only = set(args.only.split(',')) if args.only else None
    meta = {}
    for name, spec in SPECS.items():
        if only and name not in only:
            continue
        spec = dict(spec)
        if spec['T'] == 'field':
            spec['T'] = make_T_field(spec)
        rec = run_spec(hs, spec)
        rec['T'] = np.asarray(spec['T'], dtype=float) * np.ones((spec['ny'], spec['nx']))
        np.savez_compressed(os.path.join(HERE, f'{name}.npz'), **rec)
        jspec = {k: (v if not isinstance(v, np.ndarray) else 'field') for k, v in spec.items()}
        meta[name] = jspec
        print(f'{name}: steps={spec.get("steps", 0)} switches={int(rec["switches"][-1]) if len(rec["switches"]) else 0} '
              f'calls={int(rec["calls"][-1]) if len(rec["calls"]) else 0}')
    if only:
        with open(os.path.join(HERE, 'specs.json')) as f:
            merged = json.load(f)
        merged.update(meta)
        with open(os.path.join(HERE, 'specs.json'), 'w') as f:
            json.dump(merged, f, indent=1, default=float)
    else:
        hex_cases, E_theory = hexagon_kat(hs)
        np.savez_compressed(os.path.join(HERE, 'hexagon_kat.npz'), E_theory=E_theory,
                            **{f'{k}_{i}': v[i] for k, v in hex_cases.items() for i in range(3)})
        # reference Poisson selection (metres passed into a cell-unit routine): always (0,0)
        mm = hs.ASI.OOP_Square(200e-9, 16, pattern='uniform', energies=[hs.energies.DipolarEnergy()],
                               params=hs.core.SimParams(UPDATE_SCHEME='Metropolis', MULTISAMPLING_SCHEME='Poisson'))
        mm.initialize_m(random_pm1((16, 16), 5))
        route_rng(mm, PhiloxStream(5))
        sel = [np.asarray(mm.select(r=mm.calc_r(0.05))) for _ in range(3)]
        np.savez_compressed(os.path.join(HERE, 'poisson_reference.npz'), selections=np.stack(sel))
        np.savez_compressed(os.path.join(HERE, 'square_vertices.npz'), **square_vertices(hs, args.ref))
        with open(os.path.join(HERE, 'specs.json'), 'w') as f:
            json.dump(meta, f, indent=1, default=float)


if __name__ == '__main__':
    main()
