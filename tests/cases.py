"""Shared scenario plumbing for the tests: rebuilds each golden scenario for the oracle and
for the CUDA path from ``tests/golden/specs.json`` + ``tests/golden/<name>.npz``."""
from __future__ import annotations

import json
import math
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden')


def load_specs():
    with open(os.path.join(GOLDEN, 'specs.json')) as f:
        return json.load(f)


def load_fixture(name):
    with np.load(os.path.join(GOLDEN, f'{name}.npz')) as z:
        return {k: z[k] for k in z.files}


def oracle_geometry(spec):
    from oracle import geometry as G
    kind, a, nx, ny = spec['lattice'], spec['a'], spec['nx'], spec['ny']
    if kind == 'OOP_Square':
        return G.oop_square(a, nx, ny)
    if kind == 'IP_Pinwheel':
        return G.ip_pinwheel(a, nx, ny)
    if kind == 'IP_Square':
        return G.ip_square(a, nx, ny)
    if kind == 'IP_Kagome':
        return G.ip_kagome(a, nx, ny, PBC=spec.get('kw', {}).get('PBC', False))
    raise ValueError(kind)


def oracle_energies(spec):
    from oracle.hotspice_oracle import OracleDiMonopolar, OracleDipolar, OracleExchange, OracleZeeman
    out = []
    for e in spec['energies']:
        if e['type'] == 'dipolar':
            out.append(OracleDipolar(cutoff_range=e.get('cutoff', np.inf)))
        elif e['type'] == 'dimonopolar':
            out.append(OracleDiMonopolar(e.get('prefactor', 1.0), e['d'], e['small_d']))
        elif e['type'] == 'zeeman':
            out.append(OracleZeeman(e['B'], e.get('angle', 0.0)))
        elif e['type'] == 'exchange':
            out.append(OracleExchange(e['J']))
    return out


def build_oracle(name, spec=None, fx=None, **over):
    from oracle.hotspice_oracle import OracleMagnets
    spec = spec or load_specs()[name]
    fx = fx or load_fixture(name)
    g = oracle_geometry(spec)
    params = dict(spec.get('params', {}))
    params.setdefault('UPDATE_SCHEME', 'Neel')
    kw = dict(T=fx['T'], E_B=fx['E_B'], moment=spec['moment'], energies=oracle_energies(spec),
              PBC=spec.get('kw', {}).get('PBC', False), params=params, seed=spec['seed'])
    kw.update(over)
    return OracleMagnets(g, fx['m0'], **kw)


def run_relaxation(mm, spec):
    """The relax() / minimize() call a scenario ends with, if any (oracle or product)."""
    if spec.get('relax') is not None:
        mm.relax(**spec['relax'])
    if spec.get('minimize') is not None:
        mm.minimize(**spec['minimize'])


def run_io_oracle(mo, spec):
    """The oracle's input / readout loop of an 'io' scenario: one row of readouts per value."""
    from oracle.hotspice_oracle import io_input, io_read
    io = spec['io']
    outs = []
    for v in io['values']:
        io_input(mo, io['inputter'], io['params'], v)
        outs.append(io_read(mo, io['reader'], io['reader_params']))
    return np.array(outs)


def product_io_objects(mp, io):
    """The product's Inputter / OutputReader of an 'io' scenario."""
    from hotspice_b200 import io as hio
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
    else:
        ds = hio.RandomBinaryDatastream() if p.get('binary') else hio.RandomScalarDatastream()
        inp = hio.OOPSquareChessStepsInputter(ds, magnitude=p['magnitude'], magnitude_range=p['magnitude_range'],
                                              transition_range=p['transition_range'], n=p['n'], frequency=p['frequency'])
    rp = io['reader_params']
    rd = {'full': lambda: hio.FullOutputReader(mp), 'regional': lambda: hio.RegionalOutputReader(rp['nx'], rp['ny'], mp),
          'chess': lambda: hio.OOPSquareChessOutputReader(rp['nx'], rp['ny'], mp)}[io['reader']]()
    return inp, rd


def dipolar_like(mm):
    """The DipolarEnergy or DiMonopolarEnergy of an instance (oracle or product), or None."""
    for name in ('dipolar', 'dimonopolar'):
        for e in getattr(mm, 'energies', None) or getattr(mm, '_energies', ()):
            if e.shortname == name:
                return e
    return None


def rel_err(a, b):
    """Norm-wise relative error max|a-b| / max|b| (0 if both vanish)."""
    a, b = np.asarray(a, float), np.asarray(b, float)
    den = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / den) if den > 0 else float(np.max(np.abs(a - b)))
