"""FP64 CPU restatement of Hotspice's kinetic Monte Carlo hot path (test infrastructure).

ORACLE module: only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import it; the product never does. It is pinned against golden
fixtures produced by running the reference itself (``tests/golden/make_golden.py``)
with every random draw routed through :class:`oracle.philox.PhiloxStream`.

Each method cites the reference function it restates (paths relative to the
Hotspice project root). The numpy operations are deliberately the same *kind* of
full-grid array work the reference does per step, so that timing this oracle is a
fair stand-in for timing the reference's NumPy path (the reference cannot travel
to machines without its source tree).

Deviations from the reference (deliberate, each checked by the tests):
* the full dipolar recompute uses FFT convolution (FP64, ~1e-15 relative) instead of
  SciPy's direct ``convolve2d`` (hotspice/energies.py:303) so that large lattices
  initialise in seconds;
* ``select_poisson`` samples in cell units (the reference passes metres into a
  function written for cells, hotspice/core.py:564 -> hotspice/poisson.py:77,99, which
  always returns the single magnet (0,0)); ``poisson_compat=True`` reproduces the
  degenerate reference result.

Restated only in part (each part pinned by reference fixtures):
* ``minimize`` with ignore_barrier=True (with False the reference compares the
  (barrier, barrier) tuple of E_barrier() against kBT and indexes the result as one array);
* the reservoir inputs / outputs of hotspice/io.py used by the fixtures (``io_input``,
  ``io_read``): FieldInputter, PerpFieldInputter, the two checkerboard
  inputters, and the full / regional / checkerboard readers.
"""
from __future__ import annotations

import math

import numpy as np
from scipy import signal

from .geometry import Geometry, unitcell
from .philox import PhiloxStream

kB = 1.380649e-23


def lower_than(x, y, rtol=1e-10):
    """hotspice/utils.py:90-92."""
    return x < y and not np.isclose(x, y, atol=0, rtol=rtol)


def _conv_same(field, mask, PBC):
    """``signal.convolve2d(field, mask, mode='same', boundary='wrap'|'fill')``."""
    return signal.convolve2d(field, mask, mode='same', boundary='wrap' if PBC else 'fill')


# ----------------------------------------------------------------------------------------
# Energies
# ----------------------------------------------------------------------------------------
class OracleEnergy:
    def energy_switch(self, idx=None):
        """hotspice/energies.py:29-35."""
        return -2 * self.E if idx is None else -2 * self.E[idx[0], idx[1]]

    def initialize(self, mm):
        """hotspice/energies.py:37-42."""
        self.mm = mm
        self.E = np.zeros_like(mm.m)
        self.E_perp = np.zeros_like(mm.m)
        self._initialize()
        self.update()


class OracleZeeman(OracleEnergy):
    """hotspice/energies.py:86-140."""
    shortname = 'zeeman'

    def __init__(self, magnitude=0.0, angle=0.0):
        self.magnitude, self.angle = magnitude, angle

    def _initialize(self):
        mm = self.mm
        mag = np.ones(mm.shape) * self.magnitude
        ang = np.ones(mm.shape) * self.angle
        if mm.in_plane:
            bx, by = mag * np.cos(ang), mag * np.sin(ang)
            o = mm.orientation
            self.E_factor = -mm.moment * (bx * o[:, :, 0] + by * o[:, :, 1])
            self.E_factor_perp = -mm.moment * (by * o[:, :, 0] - bx * o[:, :, 1])
        else:
            self.E_factor = -mm.moment * mag
            self.E_factor_perp = np.zeros_like(mm.m)

    def set_field(self, magnitude=None, angle=None):
        """hotspice/energies.py:97-118."""
        if magnitude is not None:
            self.magnitude = magnitude
        if angle is not None:
            self.angle = angle
        self._initialize()
        self.update()

    def update(self):
        self.E = self.mm.m * self.E_factor
        if self.mm.USE_PERP_ENERGY:
            self.E_perp = self.mm.m * self.E_factor_perp

    def update_single(self, idx):
        self.E[idx[0, 0], idx[1, 0]] *= -1
        if self.mm.USE_PERP_ENERGY:
            self.E_perp[idx[0, 0], idx[1, 0]] *= -1

    def update_multiple(self, idx):
        self.E[idx[0], idx[1]] *= -1
        if self.mm.USE_PERP_ENERGY:
            self.E_perp[idx[0], idx[1]] *= -1

    @property
    def E_tot(self):
        return np.sum(self.E)


class OracleExchange(OracleEnergy):
    """hotspice/energies.py:754-791."""
    shortname = 'exchange'

    def __init__(self, J=1.0):
        self.J = J

    def _initialize(self):
        self.local_interaction = self.mm.geom.nn_mask

    def update(self):
        mm = self.mm
        if mm.in_plane:
            mx = mm.orientation[:, :, 0] * mm.m
            my = mm.orientation[:, :, 1] * mm.m
            smx = _conv_same(mx, self.local_interaction, mm.PBC)
            smy = _conv_same(my, self.local_interaction, mm.PBC)
            self.E = -self.J * (smx * mx + smy * my)
            if mm.USE_PERP_ENERGY:
                self.E_perp = -self.J * (smy * mx - smx * my)
        else:
            self.E = -self.J * (_conv_same(mm.m, self.local_interaction, mm.PBC) * mm.m)
            if mm.USE_PERP_ENERGY:
                self.E_perp = np.zeros_like(mm.m)

    def update_single(self, idx):
        self.update()

    def update_multiple(self, idx):
        self.update()

    @property
    def E_tot(self):
        return np.sum(self.E) / 2


class OracleDipolar(OracleEnergy):
    """hotspice/energies.py:143-391."""
    shortname = 'dipolar'

    def __init__(self, prefactor=1.0, decay_exponent=-3, cutoff_range=np.inf):
        self.prefactor = prefactor
        self.decay_exponent = decay_exponent
        self.cutoff_range = cutoff_range

    # -- kernel construction: hotspice/energies.py:176-288 --------------------------------
    def _initialize(self):
        self.kernels, self.kernels_perpself, self.kernels_perpother, self.kernel_index = \
            build_dipolar_kernels(self.mm, self.cutoff_range, self.decay_exponent)

    flip_perp_multiple = True   # update_multiple negates E_perp of the switched magnets

    # The interaction of a source magnet s with a target j is pref * src_s * m_j * tgt_j * K(j - s):
    # src = m * moment and tgt = moment for dipoles.
    def _src(self):
        return self.mm.m * self.mm.moment

    def _tgt(self):
        return self.mm.moment

    def update(self):
        """hotspice/energies.py:290-308 (FFT convolution instead of direct)."""
        mm = self.mm
        ux, uy = mm.unitcell
        mmom = self._src()
        tot = np.zeros_like(mm.m)
        totp = np.zeros_like(mm.m)
        for y in range(uy):
            for x in range(ux):
                n = self.kernel_index[y, x]
                if n < 0:
                    continue
                pm = np.zeros_like(mm.m)
                pm[y::uy, x::ux] = mm.m[y::uy, x::ux]
                tot += pm * signal.fftconvolve(self.kernels[n, ::-1, ::-1], mmom, mode='valid')
                if mm.USE_PERP_ENERGY:
                    totp += pm * signal.fftconvolve(self.kernels_perpself[n, ::-1, ::-1], mmom, mode='valid')
        self.E = self.prefactor * self._tgt() * tot
        if mm.USE_PERP_ENERGY:
            self.E_perp = self.prefactor * self._tgt() * totp

    def _window(self, k, y, x):
        ny, nx = self.mm.ny, self.mm.nx
        return k[ny - 1 - y:2 * ny - 1 - y, nx - 1 - x:2 * nx - 1 - x]

    def update_single(self, idx):
        """hotspice/energies.py:310-329 (called after m[idx] flipped)."""
        mm = self.mm
        y, x = int(idx[0, 0]), int(idx[1, 0])
        ux, uy = mm.unitcell
        n = self.kernel_index[y % uy, x % ux]
        if n < 0:
            return
        src, tm = self._src(), mm.m * self._tgt()
        self.E += 2 * (self.prefactor * src[y, x] * (tm * self._window(self.kernels[n], y, x)))
        self.E[y, x] *= -1
        if mm.USE_PERP_ENERGY:
            self.E_perp += 2 * (self.prefactor * src[y, x] * (tm * self._window(self.kernels_perpother[n], y, x)))
            self.E_perp[y, x] *= -1

    def update_multiple(self, idx):
        """hotspice/energies.py:331-366, including the truncated-convolution branch taken
        when more than SIMULTANEOUS_SWITCHES_CONVOLUTION_OR_SUM_CUTOFF switches share a
        sublattice (hotspice/energies.py:343-353)."""
        mm = self.mm
        perp = mm.USE_PERP_ENERGY
        self.E[idx[0], idx[1]] *= -1
        mmom = self._src()
        tm = mm.m * self._tgt()
        if perp and self.flip_perp_multiple:
            self.E_perp[idx[0], idx[1]] *= -1
        ux, uy = mm.unitcell
        sub = (idx[1] % ux) + (idx[0] % uy) * ux
        for i in np.nonzero(np.bincount(sub))[0]:
            yu, xu = divmod(int(i), ux)
            n = self.kernel_index[yu, xu]
            if n < 0:
                continue
            K = self.kernels[n]
            Kp = self.kernels_perpother[n]
            here = idx[:, sub == i]
            if here.shape[1] > mm.params['SIMULTANEOUS_SWITCHES_CONVOLUTION_OR_SUM_CUTOFF']:
                conv = truncated_window_sum(mm, here, mmom, K)
                if perp:
                    convp = truncated_window_sum(mm, here, mmom, Kp)
            else:
                conv = np.zeros_like(mm.m)
                if perp:
                    convp = np.zeros_like(mm.m)
                for j in range(here.shape[1]):
                    y, x = int(here[0, j]), int(here[1, j])
                    conv += mmom[y, x] * self._window(K, y, x)
                    if perp:
                        convp += mmom[y, x] * self._window(Kp, y, x)
            self.E += 2 * (self.prefactor * (tm * conv))
            if perp:
                self.E_perp += 2 * (self.prefactor * (tm * convp))

    @property
    def E_tot(self):
        return np.sum(self.E) / 2


def truncated_window_sum(mm, here, mmom, K):
    """Restatement of ``signal.convolve2d(switched_field, K_crop, 'same', wrap|fill)``
    (hotspice/energies.py:345-350) as a scatter of each switch's cropped window:
    the crop is K[ny-1-ky:ny+ky, nx-1-kx:nx+kx] with kx = min(R, nx-1), ky = min(R, ny-1)
    and R = REDUCED_KERNEL_SIZE; targets wrap (PBC) or are dropped (no PBC).
    R == 0 means the full kernel is used."""
    ny, nx = mm.ny, mm.nx
    R = mm.params['REDUCED_KERNEL_SIZE']
    if R:
        kx, ky = min(R, nx - 1), min(R, ny - 1)
    else:
        kx, ky = nx - 1, ny - 1
    crop = K[ny - 1 - ky:ny + ky, nx - 1 - kx:nx + kx]
    out = np.zeros_like(mm.m)
    for j in range(here.shape[1]):
        ys, xs = int(here[0, j]), int(here[1, j])
        w = mmom[ys, xs] * crop
        ty = ys - ky + np.arange(2 * ky + 1)
        tx = xs - kx + np.arange(2 * kx + 1)
        if mm.PBC:
            np.add.at(out, (np.mod(ty, ny)[:, None], np.mod(tx, nx)[None, :]), w)
        else:
            oky, okx = (ty >= 0) & (ty < ny), (tx >= 0) & (tx < nx)
            out[np.ix_(ty[oky], tx[okx])] += w[np.ix_(oky, okx)]
    return out


class OracleDiMonopolar(OracleDipolar):
    """hotspice/energies.py:394-751: every magnet is a pair of opposite magnetic charges
    q = moment / d a distance d apart along its axis; the kernel sums the four charge-charge
    terms. Targets carry q^2 and sources their bare spin (update: energies.py:684-697,
    update_single: 699-716, update_multiple: 718-751)."""
    shortname = 'dimonopolar'
    flip_perp_multiple = False  # energies.py:718-719 negates E only

    def __init__(self, prefactor=1.0, d=200e-9, small_d=200e-9):
        super().__init__(prefactor=prefactor)
        self.d = d
        self.small_d = small_d

    def _initialize(self):
        mm = self.mm
        ux, uy = mm.unitcell
        dist_uc = np.broadcast_to(np.asarray(self.d, dtype=float), (uy, ux))
        dist = np.tile(dist_uc, (math.ceil(mm.ny / uy), math.ceil(mm.nx / ux)))[:mm.ny, :mm.nx]
        self.charge_sq = (mm.moment / dist) ** 2
        self.kernels, self.kernels_perpself, self.kernels_perpother, self.kernel_index = \
            build_dimonopolar_kernels(mm, self.d, self.small_d)

    def _src(self):
        return self.mm.m

    def _tgt(self):
        return self.charge_sq


def build_dimonopolar_kernels(mm, d, small_d):
    """Monopole-pair kernels, one per occupied unit-cell site (hotspice/energies.py:406-680).

    Charges sit at +-d/2 along each magnet's original angle, on a grid of offsets from
    -(n-1) to n-1+u built from the cumulative cell spacings. For the magnet at the kernel's
    centre the kernel is sum of 1/r over its N-N and S-S pairs minus its N-S and S-N pairs
    with every other magnet (the squared distances rounded to float32, as the reference
    does), masked by the occupation; 'perp-self' rotates the centre magnet's pair by 90 deg
    with spacing small_d, 'perp-other' rotates every other magnet's. PBC folds in the 8
    neighbouring images; the result is scaled by mu0 / 4 pi = 1e-7."""
    nx, ny = mm.nx, mm.ny
    ux, uy = mm.unitcell
    scalar_d = np.ndim(d) == 0
    dist_uc = np.broadcast_to(np.asarray(d, dtype=float), (uy, ux))

    def axis(n, u, spacing):
        idx = np.arange(-(n - 1), n + u)
        c = np.zeros(idx.size)
        c[1:] = np.cumsum(np.asarray(spacing, dtype=float)[idx % n])[:-1]
        return c - c[n - 1]
    XX, YY = np.meshgrid(axis(nx, ux, mm.dx), axis(ny, uy, mm.dy))
    ry = (np.arange(XX.shape[0]) - (ny - 1)) % uy
    rx = (np.arange(XX.shape[1]) - (nx - 1)) % ux
    dist = np.full(XX.shape, float(d)) if scalar_d else dist_uc[ry[:, None], rx[None, :]]
    # the reference reads original_angles; the geometry's angles differ from them only on
    # unoccupied cells, whose kernel entries the occupation mask zeroes
    ang = mm.geom.angles[:uy, :ux][ry[:, None], rx[None, :]]
    cN_x, cS_x = XX + dist / 2 * np.cos(ang), XX - dist / 2 * np.cos(ang)
    cN_y, cS_y = YY + dist / 2 * np.sin(ang), YY - dist / 2 * np.sin(ang)
    rot = ang + np.pi / 2
    pN_x, pS_x = XX + small_d / 2 * np.cos(rot), XX - small_d / 2 * np.cos(rot)
    pN_y, pS_y = YY + small_d / 2 * np.sin(rot), YY - small_d / 2 * np.sin(rot)

    def rinv4(ax, ay, bx, by, y, x, f32):
        """1/r of NN, SS, NS, SN between the charges (ax, ay) of every magnet and the centre
        magnet (y, x) with charges (bx, by); index 0 = N, 1 = S."""
        out = []
        for i, j in ((0, 0), (1, 1), (0, 1), (1, 0)):
            dx_ = ax[i] - bx[j][y, x]
            dy_ = ay[i] - by[j][y, x]
            if i != j:
                dx_ = dx_.copy(); dy_ = dy_.copy()
                dx_[y, x] = 0.0; dy_[y, x] = 0.0
            r2 = dx_ ** 2 + dy_ ** 2
            if f32:
                r2 = r2.astype(np.float32)
            r2[r2 == 0] = np.inf
            out.append((r2 ** -0.5).astype(np.float64)[y - ny + 1:y + ny, x - nx + 1:x + nx])
        return out

    rinv, rinv_ps, rinv_po = [], [], []
    for y in range(ny - 1, ny - 1 + uy):
        for x in range(nx - 1, nx - 1 + ux):
            rinv.append(rinv4((cN_x, cS_x), (cN_y, cS_y), (cN_x, cS_x), (cN_y, cS_y), y, x, True))
            # centre magnet rotated
            sx = [cN_x.copy(), cS_x.copy()]; sy = [cN_y.copy(), cS_y.copy()]
            sx[0][y, x], sx[1][y, x] = pN_x[y, x], pS_x[y, x]
            sy[0][y, x], sy[1][y, x] = pN_y[y, x], pS_y[y, x]
            rinv_ps.append(rinv4(sx, sy, sx, sy, y, x, False))
            # every other magnet rotated
            ox = [pN_x.copy(), pS_x.copy()]; oy = [pN_y.copy(), pS_y.copy()]
            ox[0][y, x], ox[1][y, x] = cN_x[y, x], cS_x[y, x]
            oy[0][y, x], oy[1][y, x] = cN_y[y, x], cS_y[y, x]
            rinv_po.append(rinv4(ox, oy, ox, oy, y, x, False))
    occ_uc = mm.occupation[:uy, :ux]
    big = np.tile(occ_uc, (2 * math.ceil(ny / uy) + 1, 2 * math.ceil(nx / ux) + 1))
    index = -np.ones((uy, ux), dtype=int)
    Ks, Kps, Kpo = [], [], []
    n = 0
    for yu in range(uy):
        for xu in range(ux):
            if occ_uc[yu, xu] == 0:
                n += 1
                continue
            sx0 = (ux - ((nx - 1) % ux) + xu) % ux
            sy0 = (uy - ((ny - 1) % uy) + yu) % uy
            occ = big[sy0:sy0 + 2 * ny - 1, sx0:sx0 + 2 * nx - 1]
            ks = []
            for r in (rinv[n], rinv_ps[n], rinv_po[n]):
                k = r[0] * occ + r[1] * occ + (-r[2] * occ) + (-r[3] * occ)
                if mm.PBC:
                    fold_periodic_images(k, nx, ny)
                ks.append(k * 1e-7)
            n += 1
            index[yu, xu] = len(Ks)
            Ks.append(ks[0]); Kps.append(ks[1]); Kpo.append(ks[2])
    return np.asarray(Ks), np.asarray(Kps), np.asarray(Kpo), index


def build_dipolar_kernels(mm, cutoff_range=np.inf, decay_exponent=-3):
    """FP64 dipolar kernels, one per occupied unit-cell site (hotspice/energies.py:176-288).

    Returns (K, K_perpself, K_perpother, index) with K of shape (U, 2ny-1, 2nx-1) and
    index[y, x] the kernel number of unit-cell site (y, x), or -1 if that site is empty."""
    nx, ny = mm.nx, mm.ny
    ux, uy = mm.unitcell
    I = (mm.major_axis ** 2 + mm.minor_axis ** 2) / 16
    index = -np.ones((uy, ux), dtype=int)
    Ks, Kps, Kpo = [], [], []
    if mm.in_plane:
        uox = mm.orientation[:uy, :ux, 0]
        uoy = mm.orientation[:uy, :ux, 1]
    else:
        uo = mm.occupation[:uy, :ux]
    for y in range(uy):
        for x in range(ux):
            if mm.in_plane:
                ox1, oy1 = uox[y, x], uoy[y, x]
                if ox1 == 0 and oy1 == 0:
                    continue
            elif uo[y, x] == 0:
                continue
            # unit-cell phase of the first row/column of the (2ny-1, 2nx-1) kernel
            sx = (ux - ((nx - 1) % ux) + x) % ux
            sy = (uy - ((ny - 1) % uy) + y) % uy
            cols = (sx + np.arange(2 * nx - 1)) % ux
            rows = (sy + np.arange(2 * ny - 1)) % uy
            dxs = mm.dx[:ux][cols]
            dys = mm.dy[:uy][rows]
            xx = np.cumsum(np.broadcast_to(dxs[None, :], (2 * ny - 1, 2 * nx - 1)), axis=1)
            yy = np.cumsum(np.broadcast_to(dys[:, None], (2 * ny - 1, 2 * nx - 1)), axis=0)
            rrx = xx - xx[0, nx - 1]
            rry = yy - yy[ny - 1, 0]
            rr_sq = (rrx ** 2 + rry ** 2).astype(float)
            rr_sq[ny - 1, nx - 1] = np.inf
            rr_sq[rr_sq > cutoff_range ** 2] = np.inf
            rr_inv = rr_sq ** -0.5
            rinv3 = rr_inv ** (-decay_exponent)
            rinv5 = rr_inv ** (-decay_exponent + 2)
            ex = rrx * rr_inv
            ey = rry * rr_inv
            if mm.in_plane:
                ox2 = uox[rows[:, None], cols[None, :]]
                oy2 = uoy[rows[:, None], cols[None, :]]

                def ip_kernel(ax, ay, bx, by):
                    k = ax * bx * (3 * ex ** 2 - 1) + ay * by * (3 * ey ** 2 - 1) + 3 * (ex * ey) * (ax * by + ay * bx)
                    kc = ax * bx * (5 * ex ** 2 - 1) + ay * by * (5 * ey ** 2 - 1) + 5 * (ex * ey) * (ax * by + ay * bx)
                    return -rinv3 * k - 3 * I / 2 * rinv5 * kc
                K = ip_kernel(ox1, oy1, ox2, oy2)
                Kps_ = ip_kernel(-oy1, ox1, ox2, oy2)
                Kpo_ = ip_kernel(ox1, oy1, -oy2, ox2)
            else:
                o2 = uo[rows[:, None], cols[None, :]].astype(float)
                K = o2 * (rinv3 + 9 * I / 2 * rinv5)
                Kps_ = np.zeros_like(K)
                Kpo_ = np.zeros_like(K)
            if mm.PBC:
                for k in (K, Kps_, Kpo_):
                    fold_periodic_images(k, nx, ny)
            K = K * 1e-7
            Kps_ = Kps_ * 1e-7
            Kpo_ = Kpo_ * 1e-7
            index[y, x] = len(Ks)
            Ks.append(K); Kps.append(Kps_); Kpo.append(Kpo_)
    return np.asarray(Ks), np.asarray(Kps), np.asarray(Kpo), index


def fold_periodic_images(k, nx, ny):
    """Adds the 8 neighbouring periodic images into the kernel array in place
    (hotspice/energies.py:264-277): for every image shift (sy, sx) in {-1,0,1}^2 except
    (0, 0), k[d] += k_original[d - (sy*ny, sx*nx)] wherever both offsets lie in the array."""
    orig = k.copy()
    H, W = 2 * ny - 1, 2 * nx - 1
    for sy, sx in ((0, 1), (1, 1), (1, 0), (1, -1), (0, -1), (-1, -1), (-1, 0), (-1, 1)):
        # destination offset index p receives orig[p - sy*ny] (rows); valid where both in range
        ry = slice(ny, H) if sy == 1 else (slice(0, ny - 1) if sy == -1 else slice(0, H))
        rx = slice(nx, W) if sx == 1 else (slice(0, nx - 1) if sx == -1 else slice(0, W))
        sry = slice(0, ny - 1) if sy == 1 else (slice(ny, H) if sy == -1 else slice(0, H))
        srx = slice(0, nx - 1) if sx == 1 else (slice(nx, W) if sx == -1 else slice(0, W))
        k[ry, rx] += orig[sry, srx]


# ----------------------------------------------------------------------------------------
# Magnets
# ----------------------------------------------------------------------------------------
DEFAULT_PARAMS = dict(SIMULTANEOUS_SWITCHES_CONVOLUTION_OR_SUM_CUTOFF=20, REDUCED_KERNEL_SIZE=20,
                      UPDATE_SCHEME='Neel', MULTISAMPLING_SCHEME='grid',
                      ENERGY_BARRIER_METHOD='simple', METROPOLIS_TIME=False)


class OracleMagnets:
    """State and update schemes of hotspice/core.py:56-760 for one lattice instance."""

    def __init__(self, geom: Geometry, m0, *, T=300.0, E_B=0.0, moment=1e-15, energies=(),
                 PBC=False, m_perp_factor=None, major_axis=0.0, minor_axis=None, params=None,
                 seed=0, rng=None, poisson_compat=False):
        self.geom = geom
        self.nx, self.ny = geom.nx, geom.ny
        self.in_plane = geom.in_plane
        self.occupation = geom.occupation.astype(int)
        self.orientation = geom.orientation
        self.dx, self.dy = geom.dx, geom.dy
        self.x, self.y = geom.x, geom.y
        self.geom_ixx, self.geom_iyy = np.meshgrid(np.arange(self.nx), np.arange(self.ny))
        self.x_min, self.x_max = float(self.x[0]), float(self.x[-1])
        self.y_min, self.y_max = float(self.y[0]), float(self.y[-1])
        with np.errstate(divide='ignore'):
            self._occupation_inf = 1 / self.occupation
        self.nonzero = np.nonzero(self.occupation)
        self._nonzero_array = np.asarray(self.nonzero).reshape(2, -1)
        self.n = int(np.sum(self.occupation))
        self.unitcell = unitcell(geom)
        ux, uy = self.unitcell
        if PBC and (self.nx % ux or self.ny % uy):
            PBC = False  # hotspice/core.py:362-373
        self.PBC = bool(PBC)
        self.m = np.sign(np.asarray(m0, dtype=float).reshape(self.ny, self.nx)) * self.occupation
        self.T = np.ones(self.shape) * T if np.isscalar(T) else np.asarray(T, float).reshape(self.shape)
        self.E_B = np.ones(self.shape) * E_B if np.isscalar(E_B) else np.asarray(E_B, float).reshape(self.shape)
        self.moment = np.ones(self.shape) * moment if np.isscalar(moment) else np.asarray(moment, float).reshape(self.shape)
        self.m_perp_factor = float(self.in_plane if m_perp_factor is None else m_perp_factor)
        self.major_axis = major_axis
        self.minor_axis = major_axis if minor_axis is None else minor_axis
        self.params = dict(DEFAULT_PARAMS, **(params or {}))
        self.rng = PhiloxStream(seed) if rng is None else rng
        self.poisson_compat = poisson_compat
        self.t = 0.0
        self.switches = 0
        self.attempted_switches = 0
        self.energies = []
        for e in energies:
            e.initialize(self)
            self.energies.append(e)

    # -- fields --------------------------------------------------------------------------
    @property
    def shape(self):
        return (self.ny, self.nx)

    @property
    def kBT(self):
        return kB * self.T

    @property
    def beta(self):
        return 1 / self.kBT

    @property
    def USE_PERP_ENERGY(self):
        return bool(self.m_perp_factor) and self.in_plane

    @property
    def MCsteps(self):
        return self.attempted_switches / self.n

    @property
    def E(self):
        return sum(e.E for e in self.energies)

    def get_energy(self, name):
        for e in self.energies:
            if e.shortname == name:
                return e
        return None

    def update_energy(self, index=None):
        """hotspice/core.py:241-253."""
        for e in self.energies:
            if index is None:
                e.update()
            elif index[0].size == 1:
                e.update_single(index)
            elif index[0].size > 1:
                e.update_multiple(index)

    def switch_energy(self, idx=None):
        return sum(e.energy_switch(idx) for e in self.energies)

    def perp_energy(self, idx=None):
        if not self.USE_PERP_ENERGY:
            return np.zeros(self.shape) if idx is None else np.zeros(idx.shape[1])
        return self.m_perp_factor * sum(e.E_perp if idx is None else e.E_perp[idx[0], idx[1]]
                                        for e in self.energies)

    # -- barrier and update schemes ------------------------------------------------------------
    def E_barrier(self, idx=None, min_only=False):
        """hotspice/core.py:625-656."""
        with np.errstate(invalid='ignore', divide='ignore'):
            occ_inf = self._occupation_inf if idx is None else self._occupation_inf[idx[0], idx[1]]
            dE = self.switch_energy(idx) * occ_inf
            E = -dE / 2
            E_B = self.E_B if idx is None else self.E_B[idx[0], idx[1]]
        if not self.USE_PERP_ENERGY:
            if self.params['ENERGY_BARRIER_METHOD'] == 'simple':
                b = np.maximum(dE, E_B - E)
            else:
                with np.errstate(invalid='ignore', divide='ignore'):
                    inv4 = 0.25 / E_B
                    b = np.where(dE > 4 * E_B, dE, np.minimum(E_B * (dE * inv4 + 1) ** 2, dE + 4 * E_B))
            return b if min_only else (b, b)
        Ep = self.perp_energy(idx)
        b1 = np.maximum(dE, E_B + Ep - E)
        b2 = np.maximum(dE, E_B - Ep - E)
        return np.minimum(b1, b2) if min_only else (b1, b2)

    def update(self, **kw):
        """hotspice/core.py:604-622."""
        if np.any(self.T == 0):
            return None
        s = self.params['UPDATE_SCHEME']
        if s in ('Neel', 'Néel'):
            return self._update_neel(**kw)
        if s in ('Metropolis', 'Glauber'):
            return self._update_metropolis(**kw)
        if s == 'Wolff':
            return self._update_wolff()
        raise ValueError(s)

    def _update_neel(self, t_max=1, attempt_freq=1e10):
        """hotspice/core.py:679-709."""
        with np.errstate(invalid='ignore', divide='ignore', over='ignore'):
            if self.USE_PERP_ENERGY:
                b1, b2 = self.E_barrier()
                bmin = min(np.nanmin(b1), np.nanmin(b2))
                b1 = b1 - bmin
                b2 = b2 - bmin
                freq = np.exp(-b1 * self.beta) + np.exp(-b2 * self.beta)
                taus = self.rng.exponential(scale=1 / freq, size=self.shape)
                attempt_freq /= 2
            else:
                b = self.E_barrier(min_only=True)
                bmin = np.nanmin(b)
                b = b - bmin
                taus = self.rng.exponential(scale=np.exp(b * self.beta), size=self.shape)
            i = divmod(int(np.nanargmin(taus)), self.nx)
            time = taus[i] * np.exp(bmin * self.beta[i]) / attempt_freq
            self.attempted_switches += 1
            if time > t_max or np.isnan(time):
                self.t += t_max
                return None
            self.m[i] *= -1
            self.switches += 1
            self.t += float(time)
        self.update_energy(np.asarray(i).reshape(2, -1))
        return i

    def _update_metropolis(self, idx=None, Q=0.05, r=0, attempt_freq=1e10):
        """hotspice/core.py:659-677."""
        if idx is None:
            idx = self.select(r=self.calc_r(Q) if r == 0 else r)
        self.attempted_switches += idx.shape[1]
        beta = self.beta[idx[0], idx[1]]
        with np.errstate(divide='ignore', over='ignore'):
            p = np.clip(np.exp(-self.switch_energy(idx) * beta), 1e-10, 1e10)
            if self.params['METROPOLIS_TIME']:
                times = -np.log(self.rng.random(size=idx.shape[1])) / attempt_freq / self.n * \
                    np.exp(self.E_barrier(idx, min_only=True) * beta)
                self.t += np.sum(times)
        sw = idx[:, np.where(self.rng.random(size=p.shape) < p)[0]]
        if sw.shape[1] > 0:
            self.m[sw[0], sw[1]] *= -1
            self.switches += sw.shape[1]
            self.update_energy(sw)
        return sw

    def _update_wolff(self):
        """hotspice/core.py:711-718."""
        c = self.select_cluster()
        self.m[c[0], c[1]] *= -1
        self.switches += c.shape[1]
        self.attempted_switches += c.shape[1]
        self.update_energy(c)
        return c

    # -- relaxation ----------------------------------------------------------------------
    def minimize(self, ignore_barrier=True, _frac=0.3):
        """hotspice/core.py:763-797: switch, one at a time, the magnet with the most energy to
        gain; when some magnets gain more than kBT, switch a random ceil(frac n) of those n at
        once. Stops when no switch lowers the energy, or a magnet was picked a third time.
        Only ``ignore_barrier=True`` is restated: with False the reference compares the
        (barrier, barrier) tuple that E_barrier() returns."""
        if not ignore_barrier:
            raise NotImplementedError('minimize(ignore_barrier=False) indexes a (barrier, barrier) tuple')
        visited = np.zeros_like(self.m)
        while True:
            barrier = self.switch_energy()
            nob = np.where(barrier < -self.kBT)
            n = nob[0].size
            if n != 0:
                rand = self.rng.choice(n, size=math.ceil(n * _frac), replace=False)
                idx = (nob[0][rand], nob[1][rand])
            else:
                idx = divmod(int(np.argmin(barrier)), self.nx)
                if barrier[idx] >= 0:
                    break
                visited[idx] += 1
                if np.any(visited[idx] >= 3):
                    break
            idx = np.asarray(idx).reshape(2, -1)
            self.m[idx[0], idx[1]] *= -1
            self.switches += idx.shape[1]
            self.attempted_switches += idx.shape[1]
            self.update_energy(idx)

    def minimize_all(self, ignore_barrier=True, _simultaneous=False, decide=None):
        """hotspice/core.py:799-825: in a random order of the (2 ux) x (2 uy) subgrids (one
        subgrid when simultaneous), switch every magnet of the subgrid whose switch lowers the
        energy (or, with ignore_barrier False, whose switch_energy/2 + E_B < 0).
        ``decide(subset, mask)`` may replace the mask (lock-step tests)."""
        sx, sy = self.subgrid_steps(_simultaneous)
        for i in self.rng.permutation(sx * sy):
            self.minimize_subgrid(int(i), sx, sy, ignore_barrier, decide)

    def subgrid_steps(self, simultaneous=False):
        ux, uy = self.unitcell
        return (1, 1) if simultaneous else (2 * ux, 2 * uy)

    def minimize_subgrid(self, i, sx, sy, ignore_barrier=True, decide=None):
        """The body of the loop of hotspice/core.py:812-825 for subgrid number i."""
        y, x = divmod(i, sx)
        if not self.occupation[y, x]:
            return
        sub = np.asarray(np.meshgrid(np.arange(y, self.ny, sy), np.arange(x, self.nx, sx))).reshape(2, -1)
        dE = self.switch_energy(sub)
        mask = dE < 0 if ignore_barrier else dE / 2 + self.E_B[sub[0], sub[1]] < 0
        if decide is not None:
            mask = decide(sub, mask, dE)
        sel = sub[:, mask]
        if sel.size > 0:
            self.m[sel[0], sel[1]] = -self.m[sel[0], sel[1]]
            self.switches += sel.shape[1]
            self.attempted_switches += sel.shape[1]
            self.update_energy(sel)

    def relax(self, **kwargs):
        """hotspice/core.py:827-861: repeated minimize_all sweeps until a sweep switches
        nothing, the state equals the one two sweeps before (a 2-cycle), or
        int(sqrt(nx^2 + ny^2)) sweeps were made. Returns the number of sweeps."""
        n, n_max = 0, int(math.sqrt(self.nx ** 2 + self.ny ** 2))
        prev = [self.m.copy(), np.zeros_like(self.m), np.zeros_like(self.m)]
        switches = self.switches
        while not np.allclose(prev[2], prev[0]) and n < n_max:
            n += 1
            self.minimize_all(**kwargs)
            if switches == self.switches:
                break
            switches = self.switches
            prev[2] = prev[1].copy()
            prev[1] = prev[0].copy()
            prev[0] = self.m.copy()
        return n

    def calc_r(self, Q):
        """hotspice/core.py:720-733, cached per Q for the life of the instance like the
        reference's lru_cache (a later change of T or moment does not change it there either)."""
        cache = self.__dict__.setdefault('_calc_r_cache', {})
        if Q not in cache:
            r = (8e-7 * self.moment ** 2 / (Q * self.kBT)) ** (1 / 3)
            r = np.clip(r, 0, (self.x_max - self.x_min) + (self.y_max - self.y_min))
            cache[Q] = float(np.max(r))
        return cache[Q]

    # -- selection -----------------------------------------------------------------------
    def select(self, **kw):
        """hotspice/core.py:456-487 (retries until at least one occupied sample)."""
        while True:
            s = self.params['MULTISAMPLING_SCHEME']
            if s == 'single':
                pos = self.select_single()
            elif s == 'grid':
                pos = self.select_grid(**kw)
            elif s == 'Poisson':
                pos = self.select_poisson(**kw)
            elif s == 'cluster':
                pos = self.select_cluster()
            valid = np.where(self.occupation[pos[0], pos[1]])[0] if pos.size > 0 else np.zeros(0)
            if valid.size > 0:
                return pos[:, valid]

    def select_single(self, **kw):
        """hotspice/core.py:489-494."""
        i = self.rng.randint(self.n)
        return self._nonzero_array[:, i].reshape(2, -1)

    def grid_geometry(self, r):
        """Supercell size and count of hotspice/core.py:506-523."""
        ux, uy = self.unitcell
        Rx = math.ceil(r / np.min(self.dx)) - 1
        Ry = math.ceil(r / np.min(self.dy)) - 1
        Rx, Ry = ux * math.ceil(Rx / ux), uy * math.ceil(Ry / uy)
        Rx, Ry = min(Rx, self.nx), min(Ry, self.ny)
        Rx, Ry = max(Rx, 2), max(Ry, 2)
        snx, sny = self.nx // Rx + 1, self.ny // Ry + 1
        return Rx, Ry, snx, sny

    def select_grid(self, r=None, **kw):
        """hotspice/core.py:496-558 with poisson=False."""
        if r is None:
            r = self.calc_r(0.01)
        Rx, Ry, snx, sny = self.grid_geometry(r)
        ixx, iyy = np.meshgrid(np.arange(self.nx), np.arange(self.ny))
        scx = ixx[:sny:2, :snx:2].ravel()
        scy = iyy[:sny:2, :snx:2].ravel()
        nsc = scx.size
        if self.PBC:
            ox, oy = self.rng.randint(self.nx), self.rng.randint(self.ny)
        else:
            ox, oy = self.rng.randint(-Rx, Rx), self.rng.randint(-Ry, Ry)
        if Rx == self.nx:
            ox = 0
        if Ry == self.ny:
            oy = 0
        ux, uy = self.unitcell
        ddx, ddy = ox % ux, oy % uy
        occ_nz = self.occupation[ddy:ddy + Ry, ddx:ddx + Rx].nonzero()
        pick = self.rng.choice(occ_nz[0].size, nsc)
        ix = scx * Rx + occ_nz[1][pick]
        iy = scy * Ry + occ_nz[0][pick]
        if self.PBC:
            ok = (ix < max(Rx, self.nx - Rx)) & (iy < max(Ry, self.ny - Ry))
            ix, iy = ix[ok], iy[ok]
            ix = (ix + ox) % self.nx
            iy = (iy + oy) % self.ny
        else:
            ix = ix + ox
            iy = iy + oy
            ok = (ix < self.nx) & (iy < self.ny) & (ix >= 0) & (iy >= 0)
            ix, iy = ix[ok], iy[ok]
        if ix.size != 0:
            return np.asarray([iy.reshape(-1), ix.reshape(-1)])
        return self.select_single()

    def select_poisson(self, r=None, k=4, **kw):
        """hotspice/core.py:560-570 with hotspice/poisson.py:72-128 run in cell units."""
        if r is None:
            r = self.calc_r(0.01)
        if self.poisson_compat:
            return np.zeros((2, 1), dtype=int)
        r_cells = r / min(np.min(self.dx), np.min(self.dy))
        pts = poisson_disc_cells(self.nx, self.ny, r_cells, k, self.rng.random)
        if len(pts) == 0:
            return np.zeros((2, 0), dtype=int)
        p = np.asarray(pts, dtype=float).reshape(-1, 2)
        ix = nearest_index(p[:, 0], self.nx)
        iy = nearest_index(p[:, 1], self.ny)
        return np.asarray([iy, ix])

    def select_cluster(self):
        """hotspice/core.py:572-602 (exchange-only Wolff cluster)."""
        if self.get_energy('dipolar') is not None:
            raise NotImplementedError("Wolff clusters need an exchange-only system")
        ex = self.get_energy('exchange')
        if ex is None:
            raise NotImplementedError("Wolff clusters need an ExchangeEnergy")
        seed = tuple(self.select_single().flat)
        cluster = np.zeros_like(self.m)
        cluster[seed] = 1
        checked = cluster.copy()
        checked[np.where(self.m != self.m[seed])] = 1
        while np.any(front := (1 - checked) * _conv_same(cluster, ex.local_interaction, self.PBC)):
            checked[front != 0] = 1
            bond = 1 - np.exp(-2 * ex.J / self.kBT * front)
            front[self.rng.random(size=cluster.shape) > bond] = 0
            cluster[front != 0] = 1
        return np.asarray(np.where(cluster == 1))

    # -- progress ------------------------------------------------------------------------
    def progress(self, t_max=1.0, MCsteps_max=4.0, **kw):
        """hotspice/core.py:736-760."""
        t0, mc0 = self.t, self.MCsteps
        while lower_than(dt := self.t - t0, t_max) and lower_than(self.MCsteps - mc0, MCsteps_max):
            if self.params['UPDATE_SCHEME'] in ('Neel', 'Néel'):
                self.update(t_max=(t_max - dt), **kw)
            else:
                self.update(**kw)
        return self.t - t0, self.MCsteps - mc0


def nearest_index(p, n):
    """``argmin |arange(n) - p|`` with ties to the lower index (hotspice/core.py:566-567
    on a uniform grid of cell indices)."""
    p = np.asarray(p, dtype=float)
    i = np.floor(p).astype(np.int64)
    frac = p - i
    i = np.where(frac > 0.5, i + 1, i)
    return np.clip(i, 0, n - 1)


def poisson_disc_cells(width, height, r, k, random):
    """hotspice/poisson.py:72-128 (Bridson-style dart throwing, periodic distance) with
    width, height and r in cell units. ``random`` is called once per variate, in the same
    order as the reference."""
    r = r + 1
    cellsize = r / math.sqrt(2)
    rSq = r * r
    gw = math.ceil(width / cellsize)
    gh = math.ceil(height / cellsize)
    gsize = gw * gh
    grid = [None] * gsize

    def dist_sq(p, g):
        d2 = 0.0
        for dim, box in ((0, width), (1, height)):
            d = abs(p[dim] - g[dim])
            if d > box * .5:
                d -= box
            d2 += d * d
        return d2

    def fits(p, gx, gy):
        for x in range(gx - 2, gx + 3):
            for y in range(gy - 2, gy + 3):
                g = grid[(x + y * gw) % gsize]
                if g is not None and dist_sq(p, g) <= rSq:
                    return False
        return True

    p = (int(width * random()), int(height * random()))
    queue = [p]
    grid[int(p[0] / cellsize) + int(p[1] / cellsize) * gw] = p
    while queue:
        qi = int(random() * len(queue))
        qx, qy = queue.pop(qi)
        for _ in range(k):
            alpha = math.tau * random()
            d = r * math.sqrt(3 * random() + 1)
            px = qx + d * math.cos(alpha)
            py = qy + d * math.sin(alpha)
            if not (0 <= px < width and 0 <= py < height):
                continue
            q = (px, py)
            gx, gy = int(px / cellsize), int(py / cellsize)
            if not fits(q, gx, gy):
                continue
            queue.append(q)
            grid[gx + gy * gw] = q
    lim_x, lim_y = max(r, width - r), max(r, height - r)
    pts = [p for p in grid if p is not None]
    ox, oy = int(random() * width), int(random() * height)
    return [((p[0] + ox) % width, (p[1] + oy) % height) for p in pts
            if p[0] >= 0 and p[1] >= 0 and p[0] < lim_x and p[1] < lim_y]


# ----------------------------------------------------------------------------------------
# Lock-step helpers for parity tests: evaluate a step's decision without taking it, and
# apply a decision made elsewhere (teacher forcing after a near-threshold disagreement).
# ----------------------------------------------------------------------------------------
def neel_decision(mm: OracleMagnets, attempt_freq=1e10):
    """Log-domain keys of the next Néel step (same variates as _update_neel, call not
    consumed): returns (keys, taus, bmin, attempt_freq_eff). keys is +inf where unoccupied."""
    call = mm.rng.call
    u = uniform_for(mm.rng.seed, call, mm.nx * mm.ny).reshape(mm.shape)
    E1 = -np.log1p(-u)
    with np.errstate(invalid='ignore', divide='ignore', over='ignore'):
        if mm.USE_PERP_ENERGY:
            b1, b2 = mm.E_barrier()
            bmin = min(np.nanmin(b1), np.nanmin(b2))
            a1, a2 = (b1 - bmin) * mm.beta, (b2 - bmin) * mm.beta
            lo = np.minimum(a1, a2)
            logscale = lo - np.log1p(np.exp(-np.abs(a1 - a2)))
            af = attempt_freq / 2
        else:
            b = mm.E_barrier(min_only=True)
            bmin = np.nanmin(b)
            logscale = (b - bmin) * mm.beta
            af = attempt_freq
        keys = np.log(E1) + logscale
    keys = np.where(mm.occupation.astype(bool), keys, np.inf)
    return keys, np.exp(logscale) * E1, bmin, af


def uniform_for(seed, call, n):
    from .philox import uniform53
    return uniform53(seed, call, n)


def force_neel(mm: OracleMagnets, i, t_max=1.0, attempt_freq=1e10):
    """Take the Néel step with switch index ``i`` (a (y, x) tuple, or None for 'no switch
    within t_max'), consuming the step's call like _update_neel does."""
    keys, taus, bmin, af = neel_decision(mm, attempt_freq)
    mm.rng.call += 1
    mm.attempted_switches += 1
    if i is None:
        mm.t += t_max
        return None
    time = taus[i] * np.exp(bmin * mm.beta[i]) / af
    mm.m[i] *= -1
    mm.switches += 1
    mm.t += float(time)
    mm.update_energy(np.asarray(i).reshape(2, -1))
    return i


def metropolis_decision(mm: OracleMagnets, Q=0.05, r=0, attempt_freq=1e10):
    """Selection and acceptance inputs of the next Metropolis step: consumes the selection
    calls (and the METROPOLIS_TIME call), returns (idx, p, u, dt) without consuming the
    acceptance call or changing the state."""
    idx = mm.select(r=mm.calc_r(Q) if r == 0 else r)
    beta = mm.beta[idx[0], idx[1]]
    with np.errstate(divide='ignore', over='ignore'):
        p = np.clip(np.exp(-mm.switch_energy(idx) * beta), 1e-10, 1e10)
        dt = 0.0
        if mm.params['METROPOLIS_TIME']:
            times = -np.log(mm.rng.random(size=idx.shape[1])) / attempt_freq / mm.n * \
                np.exp(mm.E_barrier(idx, min_only=True) * beta)
            dt = float(np.sum(times))
    u = uniform_for(mm.rng.seed, mm.rng.call, idx.shape[1])
    return idx, p, u, dt


def force_metropolis(mm: OracleMagnets, idx, accepted_mask, dt):
    """Apply a Metropolis step whose candidates were ``idx`` and accepted ``accepted_mask``."""
    mm.rng.call += 1
    mm.attempted_switches += idx.shape[1]
    mm.t += dt
    sw = idx[:, np.asarray(accepted_mask, dtype=bool)]
    if sw.shape[1] > 0:
        mm.m[sw[0], sw[1]] *= -1
        mm.switches += sw.shape[1]
        mm.update_energy(sw)
    return sw


# ----------------------------------------------------------------------------------------
# Reservoir inputs and outputs (hotspice/io.py:193-500), the parts the fixtures exercise
# ----------------------------------------------------------------------------------------
def io_input(mm: OracleMagnets, kind, p, value):
    """One Inputter.input_single call. kind / p: 'field' (FieldInputter, io.py:221-239,
    constant or sinusoidal magnitude), 'perp' (PerpFieldInputter, io.py:270-290), 'chess'
    (OOPSquareChessFieldInputter, io.py:395-401), 'steps' (OOPSquareChessStepsInputter,
    io.py:469-500)."""
    Z = mm.get_energy('zeeman')
    if kind == 'field' and p.get('sine'):
        # io.py:228-233: the magnitude follows the sine, one update per field value
        Z.set_field(angle=(p['angle'] % math.tau) if mm.in_plane else None)
        mc0, t0 = mm.MCsteps, mm.t
        period = 1 / (1 + p['half_period'])
        while lower_than(progress := max((mm.MCsteps - mc0) / p['n'], (mm.t - t0) * p['frequency']), 1):
            Z.set_field(magnitude=p['magnitude'] * value * math.sin(progress * math.pi * 2 * period))
            mm.update(t_max=min(1 - progress, 0.05) / p['frequency'])
    elif kind == 'field':
        if mm.in_plane:
            Z.set_field(angle=p['angle'] % math.tau)
        period = 1 / (1 + p['half_period'])
        Z.set_field(magnitude=p['magnitude'] * value)
        mm.progress(t_max=1 / p['frequency'] / (2 * period), MCsteps_max=p['n'] / (2 * period))
        if not p['half_period']:
            Z.set_field(magnitude=-p['magnitude'] * value)
            mm.progress(t_max=.5 / p['frequency'], MCsteps_max=p['n'] / 2)
    elif kind == 'perp':
        angle = (p['angle'] % math.tau) + value * math.pi / 2
        for mag in [p['magnitude'], -p['magnitude']]:
            Z.set_field(magnitude=mag, angle=angle)
            if p['relax']:
                mm.minimize()
            else:
                mm.progress(t_max=0.5 / p['frequency'], MCsteps_max=p['n'])
    elif kind == 'chess':
        afm = (((mm.geom_ixx + mm.geom_iyy) % 2) * 2 - 1).astype(float)
        Z.set_field(magnitude=afm * (2 * value - 1) * p['magnitude'])
        mm.progress(t_max=1 / p['frequency'], MCsteps_max=p['n'])
    elif kind == 'steps':
        if p.get('binary'):
            mag = (2 * value - 1) * p['magnitude']
        else:
            s_ = 0.5 - p['transition_range'] / 2
            if value < s_:
                mag = -p['magnitude'] + value * p['magnitude_range'] / s_
            elif value > 1 - s_:
                mag = p['magnitude'] + (value - 1) * p['magnitude_range'] / s_
            else:
                mag = 2 * (p['magnitude'] - p['magnitude_range']) / p['transition_range'] * (value - 0.5)
        afm = ((mm.geom_ixx + mm.geom_iyy) % 2).astype(float)
        Z.set_field(magnitude=afm * mag)
        mm.progress(t_max=1 / p['frequency'], MCsteps_max=p['n'])
        Z.set_field(magnitude=(afm - 1) * mag)
        mm.progress(t_max=1 / p['frequency'], MCsteps_max=p['n'])
    else:
        raise ValueError(kind)


def io_read(mm: OracleMagnets, kind, p):
    """OutputReader.read_state: 'full' (io.py:328-332), 'regional' (io.py:346-379), 'chess'
    (io.py:417-446)."""
    if kind == 'full':
        return mm.m[mm.nonzero].astype(float)
    nxb, nyb = p['nx'], p['ny']
    rx = np.tile(np.linspace(0, nxb * (1 - 1e-15), mm.nx, dtype=int), (mm.ny, 1))
    ry = np.tile(np.linspace(0, nyb * (1 - 1e-15), mm.ny, dtype=int), (mm.nx, 1)).T
    region = rx + nxb * ry
    R = nxb * nyb
    if kind == 'chess':
        afm = ((mm.geom_ixx + mm.geom_iyy) % 2) * 2 - 1
        masked = afm * mm.m
        out = np.zeros(R)
        for r in range(R):
            out[r] = np.sum(masked[region == r]) / np.sum(mm.occupation[region == r])
        return out
    m = mm.m * mm.moment
    out = np.zeros(2 * R if mm.in_plane else R)
    norm = np.zeros(out.size)
    for i in range(out.size):
        sel = region == (i % R)
        norm[i] = np.sum(mm.occupation[sel] * mm.moment[sel])
    for r in range(R):
        sel = region == r
        if mm.in_plane:
            out[r] = np.sum((m * mm.orientation[:, :, 0])[sel])
            out[r + R] = np.sum((m * mm.orientation[:, :, 1])[sel])
        else:
            out[r] = np.sum(m[sel])
    return out / norm


# ----------------------------------------------------------------------------------------
# Vertex statistics of in-plane square ASI (examples/IP_SquareVertices.py:19-35)
# ----------------------------------------------------------------------------------------
def square_vertex_counts(m):
    """Counts (N1, N2, N3, N4) of the vertex types of an IP_Square state ``m`` (ny, nx):
    vertices are the cells with even x and y, their four magnets the neighbours left, right,
    above and below with periodic wrap (the reference's convolve2d(..., boundary='wrap')).
    N_in = m[y-1, x] + m[y, x-1] - m[y, x+1] - m[y+1, x] counts in-pointing magnets; |N_in| = 2
    is type 3, |N_in| = 4 type 4; with N_in = 0 the vertex is type 1 if
    |m[y-1, x] - m[y, x-1] + m[y, x+1] - m[y+1, x]| = 4 (the flower state), else type 2."""
    m = np.asarray(m, dtype=np.int64)
    up, down = np.roll(m, 1, axis=0), np.roll(m, -1, axis=0)        # m[y-1, x], m[y+1, x]
    left, right = np.roll(m, 1, axis=1), np.roll(m, -1, axis=1)     # m[y, x-1], m[y, x+1]
    n_in = (up + left - right - down)[::2, ::2]
    flower = (up - left + right - down)[::2, ::2]
    a_in, a_fl = np.abs(n_in), np.abs(flower)
    return (int(np.sum((a_in == 0) & (a_fl == 4))), int(np.sum((a_in == 0) & (a_fl != 4))),
            int(np.sum(a_in == 2)), int(np.sum(a_in == 4)))


def square_vertex_fractions(m):
    c = np.asarray(square_vertex_counts(m), dtype=float)
    return tuple(c / c.sum())
