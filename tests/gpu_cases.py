"""Builds the CUDA-path (product) twin of a golden scenario."""
from __future__ import annotations

import numpy as np

from cases import load_fixture, load_specs


def build_product(name, spec=None, fx=None, engine=None, **over):
    import hotspice_b200 as hs
    spec = spec or load_specs()[name]
    fx = fx or load_fixture(name)
    cls = {'OOP_Square': hs.ASI.OOP_Square, 'IP_Pinwheel': hs.ASI.IP_Pinwheel, 'IP_Square': hs.ASI.IP_Square,
           'IP_Kagome': hs.ASI.IP_Kagome}[spec['lattice']]
    energies = []
    for e in spec['energies']:
        if e['type'] == 'dipolar':
            energies.append(hs.DipolarEnergy(cutoff_range=e.get('cutoff', np.inf)))
        elif e['type'] == 'zeeman':
            energies.append(hs.ZeemanEnergy(e['B'], e.get('angle', 0.0)))
        elif e['type'] == 'exchange':
            energies.append(hs.ExchangeEnergy(e['J']))
        elif e['type'] == 'dimonopolar':
            energies.append(hs.DiMonopolarEnergy(e.get('prefactor', 1.0), e['d'], e['small_d']))
    params = dict(spec.get('params', {}))
    kw = dict(T=fx['T'], E_B=fx['E_B'], moment=spec['moment'], pattern=fx['m0'], energies=energies,
              params=hs.SimParams(**params), PBC=spec.get('kw', {}).get('PBC', False), seed=spec['seed'],
              engine=engine)
    kw.update(over)
    return cls(spec['a'], nx=spec['nx'], ny=spec['ny'], **kw)
