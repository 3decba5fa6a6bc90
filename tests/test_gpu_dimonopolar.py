"""DiMonopolarEnergy (hotspice/energies.py:394-751) on the CUDA path against the oracle.

The step-level lock-step runs of the golden scenarios (test_gpu_parity.py,
test_gpu_engine.py) already cover Néel and Metropolis with this energy; these tests pin the
update semantics directly: update_single negates E and E_perp of the switched magnet,
update_multiple negates only E (energies.py:718-719), the charge q^2 stays the one of the
initialisation when the moment changes, and the unsupported inputs are refused.
Tolerance: energies kept as FP64 sums of FP32 increments, max|dE| / max|E| <= 1e-6.
"""
import numpy as np
import pytest

from cases import dipolar_like, rel_err

pytestmark = pytest.mark.gpu
TOL = 1e-6


def _pair(n=24, PBC=False, seed=3, d=120e-9, small_d=60e-9, moment=1e-15):
    import hotspice_b200 as hs
    from oracle import geometry as G
    from oracle.hotspice_oracle import OracleDiMonopolar, OracleMagnets
    a = 300e-9
    g = G.ip_pinwheel(a, n, n)
    rng = np.random.Generator(np.random.PCG64(seed))
    m0 = (rng.integers(0, 2, size=(n, n)) * 2 - 1) * g.occupation
    mp = hs.ASI.IP_Pinwheel(a, n, T=300, E_B=5e-20, moment=moment, pattern=m0, PBC=PBC, seed=seed,
                            energies=[hs.DiMonopolarEnergy(d=d, small_d=small_d)])
    mo = OracleMagnets(g, m0, T=300.0, E_B=5e-20, moment=moment, PBC=PBC, seed=seed,
                       energies=[OracleDiMonopolar(d=d, small_d=small_d)])
    return mp, mo


def _flip(mp, mo, idx):
    m = mp.m.cpu().numpy()
    m[idx[0], idx[1]] *= -1
    mp.m = m
    mp.update_energy(index=idx)
    mo.m[idx[0], idx[1]] *= -1
    mo.update_energy(index=idx)


def _check(mp, mo, what):
    dp, do = dipolar_like(mp), dipolar_like(mo)
    assert rel_err(dp.E.cpu().numpy(), do.E) < TOL, what
    assert rel_err(dp.E_perp.cpu().numpy(), do.E_perp) < TOL, what


def _occupied(mo, k, seed):
    ys, xs = np.nonzero(mo.occupation)
    pick = np.random.Generator(np.random.PCG64(seed)).choice(ys.size, size=k, replace=False)
    return np.stack([ys[pick], xs[pick]])


@pytest.mark.parametrize('PBC', [False, True])
def test_initial_energy_and_updates(PBC):
    mp, mo = _pair(PBC=PBC)
    _check(mp, mo, 'initial')
    for s in range(4):                                     # single switches
        _flip(mp, mo, _occupied(mo, 1, 10 + s))
        _check(mp, mo, f'single {s}')
    for s, k in enumerate((2, 7, 30)):                    # multi-switch lists, E_perp keeps its sign
        _flip(mp, mo, _occupied(mo, k, 20 + s))
        _check(mp, mo, f'multiple {k}')


def test_multiple_leaves_perp_sign():
    """After a two-switch update the switched magnets' E_perp has not been negated: it equals
    the old value plus the (zero-free) interaction increments, unlike DipolarEnergy."""
    mp, mo = _pair()
    dp = dipolar_like(mp)
    idx = _occupied(mo, 2, 5)
    before = dp.E_perp.cpu().numpy()[idx[0], idx[1]]
    _flip(mp, mo, idx)
    after = dp.E_perp.cpu().numpy()[idx[0], idx[1]]
    do = dipolar_like(mo)
    assert np.allclose(after, do.E_perp[idx[0], idx[1]], rtol=1e-6, atol=0)
    assert not np.allclose(after, -before, rtol=1e-3, atol=0)


def test_moment_change_keeps_initial_charge():
    mp, mo = _pair()
    mp.moment = 2e-15
    mo.moment = np.full(mo.shape, 2e-15)
    _flip(mp, mo, _occupied(mo, 5, 7))
    _flip(mp, mo, _occupied(mo, 1, 8))
    _check(mp, mo, 'after moment change')
    # a full recompute uses the same q^2 on both sides
    mp.update_energy()
    mo.update_energy()
    _check(mp, mo, 'recompute after moment change')


def test_refusals():
    import hotspice_b200 as hs
    with pytest.raises(NotImplementedError):
        hs.ASI.IP_Pinwheel(300e-9, 16, moment=np.linspace(1e-15, 2e-15, 256).reshape(16, 16),
                           energies=[hs.DiMonopolarEnergy(d=100e-9)])
    with pytest.raises(AttributeError):          # out-of-plane lattices have no original_angles
        hs.ASI.OOP_Square(200e-9, 16, energies=[hs.DiMonopolarEnergy(d=100e-9)])
    mm = hs.ASI.IP_Pinwheel(300e-9, 16, energies=[hs.DipolarEnergy()])
    with pytest.raises(NotImplementedError):
        mm.add_energy(hs.DiMonopolarEnergy(d=100e-9))
