"""FP64 host construction of the dipolar (and two-monopole) interaction kernels and their
device windows.

Restates DipolarEnergy._initialize (hotspice/energies.py:176-288): one kernel per occupied
unit-cell site, K_s[d] for every offset d = (dy, dx) in [-(n-1), n-1]^2, built from the
distances accumulated along the (possibly non-uniform, unit-cell periodic) cell spacings,
with the finite-size ("moment of inertia") correction of Politi & Pini (2002), scaled by
mu0/4pi = 1e-7, and with the 8 neighbouring periodic images folded in when PBC is on.

For the device the kernels are stored as float32 windows of half-width (wy, wx) around
offset 0. A finite cutoff gives a small window (the bounding box of the non-zero kernel
entries). With PBC and a window narrower than half the lattice, the *unfolded* window is
stored and applied with minimum-image wrapping, which equals the folded kernel entry by
entry because at most one periodic image lies inside the cutoff.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class KernelSet:
    K: np.ndarray            # (U, 2wy+1, 2wx+1) float64
    Kps: np.ndarray          # perp-self
    Kpo: np.ndarray          # perp-other
    sub_of: np.ndarray       # (uy, ux) int32 kernel number or -1
    wx: int
    wy: int
    wrap: bool
    full: bool               # window spans every offset of the lattice
    asymmetry: float = 0.0   # see kernel_asymmetry()


def _site_axes(nx, ny, ux, uy, y, x, dx_cell, dy_cell):
    """Unit-cell phases (rows, cols) and positions (ry, rx) of every kernel offset of site
    (y, x), accumulated over the phase-shifted spacings along the full offset range."""
    H, W = 2 * ny - 1, 2 * nx - 1
    # unit-cell phase of kernel column 0 / row 0 (so that column nx-1 is site x itself)
    cols = (x - (nx - 1) + np.arange(W)) % ux
    rows = (y - (ny - 1) + np.arange(H)) % uy
    cx = np.cumsum(dx_cell[cols])
    cy = np.cumsum(dy_cell[rows])
    return rows, cols, cy - cy[ny - 1], cx - cx[nx - 1]


def _site_kernels(nx, ny, ux, uy, y, x, dx_cell, dy_cell, ori, occ, in_plane, cutoff, decay, I, hw=None):
    """Unfolded FP64 kernels (normal, perp-self, perp-other) of unit-cell site (y, x); with
    ``hw = (hy, hx)`` only the offsets |dy| <= hy, |dx| <= hx (the distances still come from
    the full-range cumulative sums, so every entry is the same as in the full kernel)."""
    rows, cols, ryv, rxv = _site_axes(nx, ny, ux, uy, y, x, dx_cell, dy_cell)
    if hw is not None:
        hy, hx = hw
        rows, ryv = rows[ny - 1 - hy:ny + hy], ryv[ny - 1 - hy:ny + hy]
        cols, rxv = cols[nx - 1 - hx:nx + hx], rxv[nx - 1 - hx:nx + hx]
        cy0, cx0 = hy, hx
    else:
        cy0, cx0 = ny - 1, nx - 1
    rx = rxv[None, :]
    ry = ryv[:, None]
    r2 = rx * rx + ry * ry
    r2[cy0, cx0] = np.inf
    r2 = np.where(r2 > cutoff * cutoff, np.inf, r2)
    rinv = r2 ** -0.5
    r3 = rinv ** (-decay)
    r5 = rinv ** (-decay + 2)
    ex, ey = rx * rinv, ry * rinv
    if not in_plane:
        o2 = occ[rows[:, None], cols[None, :]].astype(float)
        k = o2 * (r3 + 9 * I / 2 * r5)
        z = np.zeros_like(k)
        return k, z, z
    ox1, oy1 = ori[y, x]
    ox2 = ori[rows[:, None], cols[None, :], 0]
    oy2 = ori[rows[:, None], cols[None, :], 1]

    def pair(ax, ay, bx, by):
        a = ax * bx * (3 * ex * ex - 1) + ay * by * (3 * ey * ey - 1) + 3 * (ex * ey) * (ax * by + ay * bx)
        c = ax * bx * (5 * ex * ex - 1) + ay * by * (5 * ey * ey - 1) + 5 * (ex * ey) * (ax * by + ay * bx)
        return -r3 * a - 1.5 * I * r5 * c
    return pair(ox1, oy1, ox2, oy2), pair(-oy1, ox1, ox2, oy2), pair(ox1, oy1, -oy2, ox2)


def _fold(k, nx, ny):
    """Add the 8 neighbouring periodic images (array-range limited), in place."""
    src = k.copy()
    H, W = 2 * ny - 1, 2 * nx - 1
    for sy in (-1, 0, 1):
        for sx in (-1, 0, 1):
            if sy == 0 and sx == 0:
                continue
            # destination offsets d with d - (sy*ny, sx*nx) inside the array
            d_y0, d_y1 = max(0, sy * ny), min(H, H + sy * ny)
            d_x0, d_x1 = max(0, sx * nx), min(W, W + sx * nx)
            k[d_y0:d_y1, d_x0:d_x1] += src[d_y0 - sy * ny:d_y1 - sy * ny, d_x0 - sx * nx:d_x1 - sx * nx]


def build_kernels(mm, cutoff=np.inf, decay_exponent=-3) -> KernelSet:
    nx, ny = mm.nx, mm.ny
    ux, uy = mm.unitcell.x, mm.unitcell.y
    I = (mm.major_axis ** 2 + mm.minor_axis ** 2) / 16
    dx_cell = np.asarray(mm.dx[:ux], dtype=float)
    dy_cell = np.asarray(mm.dy[:uy], dtype=float)
    ori = mm.orientation[:uy, :ux] if mm.in_plane else None
    occ = mm.occupation[:uy, :ux]
    sub_of = -np.ones((uy, ux), dtype=np.int32)
    sites = []
    for y in range(uy):
        for x in range(ux):
            if mm.in_plane:
                if ori[y, x, 0] == 0 and ori[y, x, 1] == 0:
                    continue
            elif occ[y, x] == 0:
                continue
            sites.append((y, x))
    if not sites:
        raise ValueError('no occupied unit-cell site: nothing to build a dipolar kernel for')
    # with a finite cutoff, build only the offsets whose row and column distances are within it
    # (a superset of the non-zero entries), unless periodic images must be folded in
    hw = None
    if np.isfinite(cutoff):
        hy = hx = 0
        for (y, x) in sites:
            _, _, ryv, rxv = _site_axes(nx, ny, ux, uy, y, x, dx_cell, dy_cell)
            iy = np.nonzero(np.abs(ryv) <= cutoff)[0]
            ix = np.nonzero(np.abs(rxv) <= cutoff)[0]
            hy = max(hy, int(np.max(np.abs(iy - (ny - 1)))) if iy.size else 0)
            hx = max(hx, int(np.max(np.abs(ix - (nx - 1)))) if ix.size else 0)
        if not mm.PBC or (2 * hy + 1 <= ny and 2 * hx + 1 <= nx):
            hw = (hy, hx)
    ks, kps, kpo = [], [], []
    for (y, x) in sites:
        k, a, b = _site_kernels(nx, ny, ux, uy, y, x, dx_cell, dy_cell, ori, occ, mm.in_plane,
                                cutoff, decay_exponent, I, hw)
        sub_of[y, x] = len(ks)
        ks.append(k); kps.append(a); kpo.append(b)
    K, Kps, Kpo = np.asarray(ks), np.asarray(kps), np.asarray(kpo)
    cy0, cx0 = (hw[0], hw[1]) if hw is not None else (ny - 1, nx - 1)
    asym = kernel_asymmetry(K, sub_of, nx, ny, center=(cy0, cx0))
    nz = (K != 0) | (Kps != 0) | (Kpo != 0)
    rows = np.nonzero(nz.any(axis=(0, 2)))[0]
    cols = np.nonzero(nz.any(axis=(0, 1)))[0]
    wy = int(np.max(np.abs(rows - cy0))) if rows.size else 0
    wx = int(np.max(np.abs(cols - cx0))) if cols.size else 0
    finite = np.isfinite(cutoff)
    if mm.PBC and not (finite and 2 * wy + 1 <= ny and 2 * wx + 1 <= nx):
        for arr in (K, Kps, Kpo):
            for s in range(arr.shape[0]):
                _fold(arr[s], nx, ny)
        wy, wx, wrap = ny - 1, nx - 1, False
    else:
        wrap = bool(mm.PBC)
        if not finite:
            wy, wx = ny - 1, nx - 1
    sl = np.s_[:, cy0 - wy:cy0 + wy + 1, cx0 - wx:cx0 + wx + 1]
    scale = 1e-7  # mu0 / 4 pi
    return KernelSet(K[sl] * scale, Kps[sl] * scale, Kpo[sl] * scale, sub_of, wx, wy, wrap,
                     wy == ny - 1 and wx == nx - 1 and not wrap, asym)


def kernel_asymmetry(K, sub_of, nx, ny, center=None):
    """max |K_s(d) - K_s'(-d)| / max |K| over all sites s and offsets d, s' the site at d.

    The interaction of two magnets must not depend on which one is the kernel's centre, and
    it does not, except through rounding: distances come from cumulative sums of the cell
    spacings (as in the reference), so r(d) and r(-d) can differ in the last bit, and a pair
    at exactly the cutoff radius can be kept one way and dropped the other. Incremental
    updates use the switched magnet's kernel while a full recompute uses the target's, so a
    non-zero value means the incremental energies drift from a full recompute by design (the
    reference drifts identically)."""
    uy, ux = sub_of.shape
    H, W = K.shape[1], K.shape[2]
    cy0, cx0 = center if center is not None else (ny - 1, nx - 1)
    flip = K[:, ::-1, ::-1]
    worst = 0.0
    for ys in range(uy):
        for xs in range(ux):
            s = sub_of[ys, xs]
            if s < 0:
                continue
            rows = (ys - cy0 + np.arange(H)) % uy
            cols = (xs - cx0 + np.arange(W)) % ux
            tgt = sub_of[rows[:, None], cols[None, :]]
            other = np.where(tgt >= 0, flip[np.clip(tgt, 0, None), np.arange(H)[:, None], np.arange(W)[None, :]], 0.0)
            worst = max(worst, float(np.max(np.abs(K[s] - other))))
    den = float(np.max(np.abs(K)))
    return worst / den if den > 0 else 0.0


def _charge_axis(n, u, spacing):
    """Positions of the big-grid columns -(n-1) .. n-1+u relative to column 0, accumulated from
    the per-cell spacings as hotspice/energies.py:419-429 does (same summation order)."""
    idx = np.arange(-(n - 1), n + u)
    c = np.zeros(idx.size)
    c[1:] = np.cumsum(np.asarray(spacing, dtype=float)[idx % n])[:-1]
    return c - c[n - 1]


def _inv_distances(ax, ay, cx, cy, f32):
    """1/r between the charges (ax[i], ay[i]) of every window cell and the centre charges
    (cx[j], cy[j]) for the pairs NN, SS, NS, SN (index 0 = north, 1 = south). The cross pairs
    of the centre magnet with itself are excluded, coincident charges give 0 (r^2 = 0 is
    replaced by infinity), and ``f32`` rounds r^2 to float32 first, as the reference does for
    the parallel kernel (hotspice/energies.py:494-513)."""
    H, W = ax[0].shape
    out = []
    for i, j in ((0, 0), (1, 1), (0, 1), (1, 0)):
        ddx = ax[i] - cx[j]
        ddy = ay[i] - cy[j]
        if i != j:
            ddx[H // 2, W // 2] = 0.0
            ddy[H // 2, W // 2] = 0.0
        r2 = ddx ** 2 + ddy ** 2
        if f32:
            r2 = r2.astype(np.float32)
        r2[r2 == 0] = np.inf
        out.append((r2 ** -0.5).astype(np.float64))
    return out


def build_dimonopolar_kernels(mm, d, small_d, scale=1.0) -> KernelSet:
    """Kernels of the two-monopole (dumbbell) interaction, hotspice/energies.py:406-680.

    Each magnet is a pair of charges +q, -q at +-d/2 along its original angle. The kernel of
    unit-cell site s at offset o is 1e-7 * occ(s + o) * (1/r_NN + 1/r_SS - 1/r_NS - 1/r_SN)
    between the magnet at o and the one at the centre; 'perp-self' turns the centre pair by
    90 degrees with spacing ``small_d``, 'perp-other' turns every other pair instead. With PBC
    the 8 neighbouring images are folded in, so the window is always the full lattice.
    ``scale`` multiplies every entry (the energy class folds the charge factor 1/d^2 in, so
    the device field stays m * moment). The distances are taken on each centre's window
    only; every entry is computed by the same operations as in the reference's full grid."""
    nx, ny = mm.nx, mm.ny
    ux, uy = mm.unitcell.x, mm.unitcell.y
    H, W = 2 * ny - 1, 2 * nx - 1
    xl = _charge_axis(nx, ux, mm.dx)
    yl = _charge_axis(ny, uy, mm.dy)
    ang_uc = np.asarray(mm.original_angles, dtype=float)[:uy, :ux]
    occ_uc = np.asarray(mm.occupation)[:uy, :ux]
    sub_of = -np.ones((uy, ux), dtype=np.int32)
    ks, kps, kpo = [], [], []
    for yu in range(uy):
        for xu in range(ux):
            if occ_uc[yu, xu] == 0:
                continue
            # window of the centre magnet at big-grid (ny-1+yu, nx-1+xu): big rows yu .. yu+H-1
            rows, cols = np.arange(yu, yu + H), np.arange(xu, xu + W)
            XX, YY = np.meshgrid(xl[cols], yl[rows])
            ang = ang_uc[((rows - (ny - 1)) % uy)[:, None], ((cols - (nx - 1)) % ux)[None, :]]
            cos_a, sin_a = np.cos(ang), np.sin(ang)
            cos_p, sin_p = np.cos(ang + np.pi / 2), np.sin(ang + np.pi / 2)
            par_x = (XX + d / 2 * cos_a, XX - d / 2 * cos_a)
            par_y = (YY + d / 2 * sin_a, YY - d / 2 * sin_a)
            perp_x = (XX + small_d / 2 * cos_p, XX - small_d / 2 * cos_p)
            perp_y = (YY + small_d / 2 * sin_p, YY - small_d / 2 * sin_p)
            c = (ny - 1, nx - 1)
            # parallel: every pair along its axis
            r_par = _inv_distances(par_x, par_y, [a[c] for a in par_x], [a[c] for a in par_y], True)
            # perp-self: the centre pair turned (spacing small_d)
            sx, sy = [a.copy() for a in par_x], [a.copy() for a in par_y]
            for k in (0, 1):
                sx[k][c], sy[k][c] = perp_x[k][c], perp_y[k][c]
            r_ps = _inv_distances(sx, sy, [a[c] for a in sx], [a[c] for a in sy], False)
            # perp-other: every pair but the centre one turned
            ox, oy = [a.copy() for a in perp_x], [a.copy() for a in perp_y]
            for k in (0, 1):
                ox[k][c], oy[k][c] = par_x[k][c], par_y[k][c]
            r_po = _inv_distances(ox, oy, [a[c] for a in ox], [a[c] for a in oy], False)
            sy0 = (uy - ((ny - 1) % uy) + yu) % uy
            sx0 = (ux - ((nx - 1) % ux) + xu) % ux
            occ = occ_uc[((sy0 + np.arange(H)) % uy)[:, None], ((sx0 + np.arange(W)) % ux)[None, :]].astype(np.float64)
            out = []
            for r in (r_par, r_ps, r_po):
                k = r[0] * occ + r[1] * occ + (-r[2] * occ) + (-r[3] * occ)
                if mm.PBC:
                    _fold(k, nx, ny)
                k *= 1e-7  # mu0 / 4 pi
                out.append(k * scale)
            sub_of[yu, xu] = len(ks)
            ks.append(out[0]); kps.append(out[1]); kpo.append(out[2])
    if not ks:
        raise ValueError('no occupied unit-cell site: nothing to build a monopole kernel for')
    K, Kps, Kpo = np.asarray(ks), np.asarray(kps), np.asarray(kpo)
    asym = kernel_asymmetry(K, sub_of, nx, ny)
    return KernelSet(K, Kps, Kpo, sub_of, nx - 1, ny - 1, False, True, asym)
