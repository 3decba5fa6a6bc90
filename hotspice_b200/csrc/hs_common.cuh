// Shared device helpers of the sm_100a kinetic Monte Carlo kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#include "../../include/hotspice_b200.h"

#define HS_DEV __device__ __forceinline__
#define HS_HD __host__ __device__

// ---------------------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC'11). Counter = (element, call_lo, call_hi, 0),
// key = (seed_lo, seed_hi); u53 = ((w0 >> 5) * 2^26 + (w1 >> 6)) * 2^-53.
// Must stay bit-identical to oracle/philox.py.
// ---------------------------------------------------------------------------------------
struct HsU4 { uint32_t x, y, z, w; };

HS_DEV HsU4 hs_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        // one 32 x 32 -> 64-bit product per word gives both halves
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t lo0 = (uint32_t)p0, hi0 = (uint32_t)(p0 >> 32);
        const uint32_t lo1 = (uint32_t)p1, hi1 = (uint32_t)(p1 >> 32);
        const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    return HsU4{c0, c1, c2, c3};
}

// Philox round keys of a seed: (k0 + r 0x9E3779B9, k1 + r 0xBB67AE85), r = 0..9. A loop over
// many elements with one seed computes them once (they are warp-uniform).
struct HsRoundKeys { uint32_t k0[10], k1[10]; };
HS_DEV HsRoundKeys hs_round_keys(uint64_t seed) {
    HsRoundKeys R;
    uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#pragma unroll
    for (int r = 0; r < 10; ++r) { R.k0[r] = k0; R.k1[r] = k1; k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    return R;
}
// hs_philox with precomputed round keys (the same rounds, bit for bit).
HS_DEV HsU4 hs_philox_rk(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, const HsRoundKeys &R) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t lo0 = (uint32_t)p0, hi0 = (uint32_t)(p0 >> 32);
        const uint32_t lo1 = (uint32_t)p1, hi1 = (uint32_t)(p1 >> 32);
        const uint32_t n0 = hi1 ^ c1 ^ R.k0[r], n2 = hi0 ^ c3 ^ R.k1[r];
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
    }
    return HsU4{c0, c1, c2, c3};
}

HS_DEV double hs_u53_of(HsU4 w) {
    const double hi = (double)(w.x >> 5), lo = (double)(w.y >> 6);
    return (hi * 67108864.0 + lo) * (1.0 / 9007199254740992.0);
}

HS_DEV HsU4 hs_philox_at(uint64_t seed, uint64_t call, uint32_t element) {
    return hs_philox(element, (uint32_t)call, (uint32_t)(call >> 32), 0u, (uint32_t)seed, (uint32_t)(seed >> 32));
}

HS_DEV double hs_u53(uint64_t seed, uint64_t call, uint32_t element) {
    return hs_u53_of(hs_philox_at(seed, call, element));
}

// A float lower bound of u53 from the first word alone: (w0 >> 8) 2^-24 <= (w0 >> 5) 2^-27 <= u53.
HS_DEV float hs_u24_low(HsU4 w) { return (float)(w.x >> 8) * 5.9604644775390625e-08f; }

// Exponential variate E1 = -log1p(-u), accurate for small u and for u near 1.
HS_DEV double hs_exp1_f64(double u) { return -log1p(-u); }

// log(E1) in single precision (used only for the argmin key).
HS_DEV float hs_log_exp1_f32(double u) {
    float e1;
    if (u < 0.5) e1 = -log1pf(-(float)u);
    else e1 = -logf((float)(1.0 - u));
    return logf(e1);
}

// Cells of the Poisson-disc background grid (hotspice/poisson.py:78-83 in cell units), as a
// double so that no radius overflows it; the entry points refuse grids above HS_POISSON_GRID_MAX.
constexpr int HS_POISSON_GRID_MAX = 1 << 28;
HS_HD inline double hs_poisson_grid_cells(const HsLattice &L, const HsGridPlan &P) {
    const double r = P.r_cells + 1.0, cs = r / sqrt(2.0);
    return ceil(L.nx / cs) * ceil(L.ny / cs);
}

// ---------------------------------------------------------------------------------------
// Lattice helpers
// ---------------------------------------------------------------------------------------
// Sublattice of cell (y, x), both >= 0; -1 for a unit-cell site without a magnet. Unit cells
// whose sides are powers of two (1, 2 and 4 cells for every lattice here) take masks instead of
// integer divisions (the same remainders for non-negative coordinates).
HS_DEV int hs_sub(const HsLattice &L, int y, int x) {
    const int ry = (L.uy & (L.uy - 1)) == 0 ? (y & (L.uy - 1)) : y % L.uy;
    const int rx = (L.ux & (L.ux - 1)) == 0 ? (x & (L.ux - 1)) : x % L.ux;
    return L.sub_of[ry * L.ux + rx];
}

HS_DEV int hs_wrap(int v, int n) { v %= n; return v < 0 ? v + n : v; }

// Device wall clock (PTX %globaltimer), nanoseconds.
HS_DEV unsigned long long hs_globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Minimum-image offset of d for period n, in [-(n/2), n - n/2 - 1].
HS_DEV int hs_minimage(int d, int n) {
    int r = hs_wrap(d, n);
    return (2 * r >= n) ? r - n : r;
}

// Kernel value of sublattice `s` at (non-wrapped) offset (dy, dx), both in [-(n-1), n-1].
// Window storage: (2wy+1, 2wx+1), centre at (wy, wx). In wrap mode the stored window is the
// minimum-image crop of the periodically folded kernel.
HS_DEV float hs_kval(const HsLattice &L, const float *K, int s, int dy, int dx) {
    if (L.dip_wrap) { dy = hs_minimage(dy, L.ny); dx = hs_minimage(dx, L.nx); }
    if (dy < -L.dip_wy || dy > L.dip_wy || dx < -L.dip_wx || dx > L.dip_wx) return 0.f;
    const int64_t W = (int64_t)(2 * L.dip_wx + 1), H = (int64_t)(2 * L.dip_wy + 1);
    return __ldg(K + (int64_t)s * H * W + (int64_t)(dy + L.dip_wy) * W + (dx + L.dip_wx));
}

// Exchange energy at cell (y, x) from the spins (hotspice/energies.py:771-781), convolution
// semantics with 'wrap' (PBC) or zero fill. Returns E and, for in-plane lattices, E_perp.
HS_DEV void hs_exchange_at(const HsLattice &L, int y, int x, double &E, double &Ep) {
    const int ch = L.nn_h / 2, cw = L.nn_w / 2;
    E = 0.0; Ep = 0.0;
    const int64_t i = (int64_t)y * L.nx + x;
    if (!L.in_plane) {
        int s = 0;
        for (int a = 0; a < L.nn_h; ++a)
            for (int b = 0; b < L.nn_w; ++b) {
                const int w = L.nn[a * L.nn_w + b];
                if (!w) continue;
                int yy = y + ch - a, xx = x + cw - b;
                if (L.pbc) { yy = hs_wrap(yy, L.ny); xx = hs_wrap(xx, L.nx); }
                else if (yy < 0 || yy >= L.ny || xx < 0 || xx >= L.nx) continue;
                s += w * (int)__ldcg(L.m + (int64_t)yy * L.nx + xx);
            }
        E = -L.J * ((double)s * (double)__ldcg(L.m + i));
    } else {
        double smx = 0.0, smy = 0.0;
        for (int a = 0; a < L.nn_h; ++a)
            for (int b = 0; b < L.nn_w; ++b) {
                const int w = L.nn[a * L.nn_w + b];
                if (!w) continue;
                int yy = y + ch - a, xx = x + cw - b;
                if (L.pbc) { yy = hs_wrap(yy, L.ny); xx = hs_wrap(xx, L.nx); }
                else if (yy < 0 || yy >= L.ny || xx < 0 || xx >= L.nx) continue;
                const int64_t j = (int64_t)yy * L.nx + xx;
                const double mj = (double)__ldcg(L.m + j);
                smx += w * (double)L.orient[2 * j] * mj;
                smy += w * (double)L.orient[2 * j + 1] * mj;
            }
        const double mi = (double)__ldcg(L.m + i);
        const double mx = (double)L.orient[2 * i] * mi, my = (double)L.orient[2 * i + 1] * mi;
        E = -L.J * (smx * mx + smy * my);
        Ep = -L.J * (smy * mx - smx * my);
    }
}

// Total energy E and perpendicular energy (before m_perp_factor) of cell i.
HS_DEV void hs_energy_at(const HsLattice &L, int y, int x, double &E, double &Ep) {
    const int64_t i = (int64_t)y * L.nx + x;
    E = 0.0; Ep = 0.0;
    if (L.has_dipolar) {
        E += (double)__ldcg(L.E_dip + i);
        if (L.use_perp) Ep += (double)__ldcg(L.E_dip_perp + i);
    }
    if (L.zee) {   // the Zeeman factors are read-only during a launch
        const double mi = (double)__ldcg(L.m + i);
        E += mi * (double)__ldg(L.zee + i);
        if (L.use_perp) Ep += mi * (double)__ldg(L.zee_perp + i);
    }
    if (L.has_exchange) {
        double e, ep;
        hs_exchange_at(L, y, x, e, ep);
        E += e;
        if (L.use_perp) Ep += ep;
    }
}

HS_DEV double hs_beta(const HsLattice &L, int64_t i) {
    return L.beta_uniform > 0.0 ? L.beta_uniform : (double)L.beta[i];
}

// Effective barrier(s) of hotspice/core.py:625-656 for one occupied cell.
HS_DEV void hs_barriers(const HsLattice &L, int y, int x, double &b1, double &b2) {
    double E, Ep;
    hs_energy_at(L, y, x, E, Ep);
    const int64_t i = (int64_t)y * L.nx + x;
    const double dE = -2.0 * E;      // switch_energy
    const double Ecur = -dE / 2.0;    // E = -delta_E/2
    const double EB = (double)L.E_B[i];
    if (!L.use_perp) {
        double b;
        if (L.barrier_method == HS_BARRIER_SIMPLE) {
            b = fmax(dE, EB - Ecur);
        } else {
            const double inv4 = 0.25 / EB;
            const double q = dE * inv4 + 1.0;
            b = (dE > 4.0 * EB) ? dE : fmin(EB * q * q, dE + 4.0 * EB);
        }
        b1 = b2 = b;
    } else {
        const double Ept = L.m_perp_factor * Ep;
        b1 = fmax(dE, (EB + Ept) - Ecur);
        b2 = fmax(dE, (EB - Ept) - Ecur);
    }
}

// progress() stop rule of hotspice/core.py:753-760 with utils.lower_than (rtol 1e-10).
HS_DEV bool hs_lower_than(double x, double y) {
    // numpy.isclose treats an infinite y as close only to itself
    if (isinf(y)) return x < y;
    return x < y && !(fabs(x - y) <= 1e-10 * fabs(y));
}

HS_DEV bool hs_progress_continue(const HsCounters *C, int n_occ) {
    if (!C->progress) return true;
    const double dt = C->t - C->t0;
    const double dmc = (double)C->attempted / (double)n_occ - C->mc0;
    return hs_lower_than(dt, C->t_max) && hs_lower_than(dmc, C->mc_max);
}

// Arg-min helpers: smaller key wins, ties go to the smaller index (numpy nanargmin). A Néel
// candidate also carries its two barriers and, when the scan loaded them, its moment mm and
// spin m (m = 0: not carried), so the step's decision needs no reload of them.
struct HsKeyIdx { double key; int idx; double b1, b2; float mm; int m; };
HS_DEV HsKeyIdx hs_kmin(HsKeyIdx a, HsKeyIdx b) {
    if (b.idx < 0) return a;
    if (a.idx < 0) return b;
    if (b.key < a.key || (b.key == a.key && b.idx < a.idx)) return b;
    return a;
}
HS_DEV HsKeyIdx hs_warp_kmin(HsKeyIdx v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        HsKeyIdx w;
        w.key = __shfl_xor_sync(0xffffffffu, v.key, o);
        w.idx = __shfl_xor_sync(0xffffffffu, v.idx, o);
        w.b1 = __shfl_xor_sync(0xffffffffu, v.b1, o);
        w.b2 = __shfl_xor_sync(0xffffffffu, v.b2, o);
        w.mm = __shfl_xor_sync(0xffffffffu, v.mm, o);
        w.m = __shfl_xor_sync(0xffffffffu, v.m, o);
        v = hs_kmin(v, w);
    }
    return v;
}
