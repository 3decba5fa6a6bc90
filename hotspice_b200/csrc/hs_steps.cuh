// Step bodies shared by the standalone step kernels and the persistent cluster engine.
#pragma once

#include "hs_common.cuh"

// ---- dipolar window helpers ----------------------------------------------------------


struct SwInfo { int y, x, mode, sub; float mm; };

// Does the window of switch (ys, mode) reach rows [t0, t0 + tn) (1-D test, axis length n)?
HS_DEV bool hs_axis_overlap(int s, int half, int wrap, int n, int t0, int tn) {
    if (wrap) {
        if (2 * half + 1 >= n) return true;
        const int ws = s - half;
        return hs_wrap(t0 - ws, n) <= 2 * half || hs_wrap(ws - t0, n) < tn;
    }
    return !(s + half < t0 || s - half >= t0 + tn);
}

// Window half-width and wrap flag of a switch along one axis.
HS_DEV void hs_window(const HsLattice &L, int mode, bool yaxis, int &half, int &wrap) {
    const int n = yaxis ? L.ny : L.nx;
    if (mode) {
        half = L.trunc_size ? min(L.trunc_size, n - 1) : n - 1;
        wrap = L.pbc;
    } else {
        half = yaxis ? L.dip_wy : L.dip_wx;
        wrap = L.dip_wrap;
    }
}

// Sum of kernel values that switch `w` contributes to target (y, x).
HS_DEV void hs_contrib(const HsLattice &L, const SwInfo &w, int y, int x, float &acc, float &accp) {
    if (!w.mode) {
        const int dy = y - w.y, dx = x - w.x;
        acc += w.mm * hs_kval(L, L.K, w.sub, dy, dx);
        if (L.use_perp) accp += w.mm * hs_kval(L, L.Kpo, w.sub, dy, dx);
        return;
    }
    const int ky = L.trunc_size ? min(L.trunc_size, L.ny - 1) : L.ny - 1;
    const int kx = L.trunc_size ? min(L.trunc_size, L.nx - 1) : L.nx - 1;
    int dys[2], dxs[2], ny_ = 0, nx_ = 0;
    if (L.pbc) {
        const int d0y = hs_wrap(y - w.y, L.ny), d0x = hs_wrap(x - w.x, L.nx);
        if (d0y <= ky) dys[ny_++] = d0y;
        if (d0y - L.ny >= -ky) dys[ny_++] = d0y - L.ny;
        if (d0x <= kx) dxs[nx_++] = d0x;
        if (d0x - L.nx >= -kx) dxs[nx_++] = d0x - L.nx;
    } else {
        const int dy = y - w.y, dx = x - w.x;
        if (dy >= -ky && dy <= ky) dys[ny_++] = dy;
        if (dx >= -kx && dx <= kx) dxs[nx_++] = dx;
    }
    for (int a = 0; a < ny_; ++a)
        for (int b = 0; b < nx_; ++b) {
            acc += w.mm * hs_kval(L, L.K, w.sub, dys[a], dxs[b]);
            if (L.use_perp) accp += w.mm * hs_kval(L, L.Kpo, w.sub, dys[a], dxs[b]);
        }
}


// ---- Metropolis ------------------------------------------------------------------------

constexpr int MT = 1024;              // threads of the step CTA
constexpr int MAX_RETRY = 1 << 14;    // bound on select() retries before reporting

struct MetroScratch {
    int32_t *py, *px;                  // candidate positions (capacity cap)
    int32_t *grid;                     // Poisson background grid (gsz)
    double  *ptx, *pty;                // Poisson points (gsz)
    int32_t *queue;                    // Poisson active list (gsz)
    int32_t cap, gsz;
};

HS_DEV int block_excl_scan(int flag, int *warp_tot, int &total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned bal = __ballot_sync(0xffffffffu, flag);
    if (lane == 0) warp_tot[warp] = __popc(bal);
    __syncthreads();
    if (warp == 0) {
        int v = lane < (int)(blockDim.x >> 5) ? warp_tot[lane] : 0;
        int incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) { int t = __shfl_up_sync(0xffffffffu, incl, o); if (lane >= o) incl += t; }
        if (lane < (int)(blockDim.x >> 5)) warp_tot[lane] = incl - v;
        if (lane == 31) warp_tot[32] = incl;
    }
    __syncthreads();
    const int pre = warp_tot[warp] + __popc(bal & ((1u << lane) - 1u));
    total = warp_tot[32];
    __syncthreads();
    return pre;
}

// Stable in-place compaction of (py, px)[0..n) keeping entries for which keep(y, x) holds.
template <typename F>
HS_DEV int block_compact(int32_t *py, int32_t *px, int n, F keep, int *warp_tot) {
    int out = 0;
    for (int base = 0; base < n; base += blockDim.x) {
        const int i = base + threadIdx.x;
        int y = 0, x = 0, f = 0;
        if (i < n) { y = py[i]; x = px[i]; f = keep(y, x) ? 1 : 0; }
        int tot;
        const int pre = block_excl_scan(f, warp_tot, tot);
        if (f) { py[out + pre] = y; px[out + pre] = x; }
        out += tot;
        __syncthreads();
    }
    return out;
}

HS_DEV int pymod(int a, int n) { int r = a % n; return r < 0 ? r + n : r; }

// Work arrays of the Poisson-disc sampler: shared memory when they fit, else the step's scratch.
struct PoissonMem {
    int32_t *grid;     // background grid: point index per cell, or -1
    double *ptx, *pty; // points
    int32_t *queue;    // active list
};

// Bytes of the work arrays for a grid of gsz cells (one point per cell at most).
HS_HD inline int64_t hs_poisson_mem_bytes(int64_t gsz) { return 24 * gsz + 64; }

HS_DEV PoissonMem poisson_mem_in(void *base, int gsz) {
    char *p = reinterpret_cast<char *>(base);
    PoissonMem M;
    M.ptx = reinterpret_cast<double *>(p);
    M.pty = M.ptx + gsz;
    M.grid = reinterpret_cast<int32_t *>(M.pty + gsz);
    M.queue = M.grid + gsz;
    return M;
}

// Poisson-disc dart throwing in cell units (hotspice/poisson.py:72-128 restated in cells),
// executed by one warp. Returns the number of points written to (S.py, S.px) as nearest cell
// indices and advances `call` by the variates consumed.
// Bridson's loop is sequential over active points, but the k tries of one active point always
// consume 1 + 2k variates (queue pick, then angle and distance of each try), so the warp
// evaluates the k candidates at once (lane t: try t) and their 5x5-cell conflict checks against
// the existing points in parallel, then resolves them in try order: try t is accepted if it is
// in bounds, conflicts with no existing point, and with no earlier accepted try whose cell is
// among the 25 it checks. Two points in one cell always conflict (the cell diagonal is r), so an
// accepted try never hides an existing point from a later try: the accepted set is the one the
// sequential loop would build, in the same order, with the same variates.
HS_DEV int poisson_warp(const HsLattice &L, const HsGridPlan &P, const MetroScratch &S, const PoissonMem &M,
                        uint64_t &call, int *status) {
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    const double width = L.nx, height = L.ny;
    const double r = P.r_cells + 1.0;
    const double cs = r / sqrt(2.0);
    const double rSq = r * r;
    const int gw = (int)ceil(width / cs), gh = (int)ceil(height / cs);
    const int gsz = gw * gh;
    const int K = P.poisson_k;
    if (gsz > S.gsz || K < 1 || 25 * K > 32 * 32) { if (lane == 0) *status |= HS_ST_POISSON_OVERFLOW; return 0; }
    for (int g = lane; g < gsz; g += 32) M.grid[g] = -1;
    __syncwarp();
    auto rnd_at = [&](uint64_t c) { return hs_u53(L.seed, c, 0u); };
    const double p0x = (double)(int)(width * rnd_at(call));
    const double p0y = (double)(int)(height * rnd_at(call + 1));
    call += 2;
    int npts = 1, nq = 1;
    if (lane == 0) { M.ptx[0] = p0x; M.pty[0] = p0y; M.queue[0] = 0; M.grid[(int)(p0x / cs) + (int)(p0y / cs) * gw] = 0; }
    __syncwarp();
    auto conflicts = [&](double px, double py, int g) {   // the distance rule of the grid check
        double dx = fabs(px - M.ptx[g]), dy = fabs(py - M.pty[g]);
        if (dx > width * 0.5) dx -= width;
        if (dy > height * 0.5) dy -= height;
        return (dx * dx + dy * dy) <= rSq;
    };
    bool overflow = false;
    while (nq > 0 && !overflow) {
        const int qi = (int)(rnd_at(call) * nq);
        const uint64_t cbase = call + 1;
        call += 1 + 2 * (uint64_t)K;
        const int q = M.queue[qi];
        // list.pop(qi): shift the tail left, preserving order
        for (int j = qi + lane; j < nq - 1; j += 32) {
            const int v = M.queue[j + 1];
            __syncwarp(__activemask());
            M.queue[j] = v;
        }
        __syncwarp();
        nq -= 1;
        const double qx = M.ptx[q], qy = M.pty[q];
        // candidates of the k tries, one per lane
        double px = 0.0, py = 0.0;
        int gx = 0, gy = 0, inb = 0;
        if (lane < K) {
            const double alpha = 6.283185307179586 * rnd_at(cbase + 2 * lane);
            const double d = r * sqrt(3.0 * rnd_at(cbase + 2 * lane + 1) + 1.0);
            px = qx + d * cos(alpha);
            py = qy + d * sin(alpha);
            inb = 0.0 <= px && px < width && 0.0 <= py && py < height;
            if (inb) { gx = (int)(px / cs); gy = (int)(py / cs); }
        }
        // conflicts with existing points: task id = 25 t + c (cell c of try t's 5x5 neighbourhood)
        unsigned cmask = 0u;
        for (int base = 0; base < 25 * K; base += 32) {
            const int id = base + lane;
            const int t = id < 25 * K ? id / 25 : 0, c = id - 25 * t;
            const double tx = __shfl_sync(0xffffffffu, px, t), ty = __shfl_sync(0xffffffffu, py, t);
            const int tgx = __shfl_sync(0xffffffffu, gx, t), tgy = __shfl_sync(0xffffffffu, gy, t);
            const int tin = __shfl_sync(0xffffffffu, inb, t);
            if (id < 25 * K && tin) {
                const int xx = tgx - 2 + c / 5, yy = tgy - 2 + c % 5;
                const int g = M.grid[pymod(xx + yy * gw, gsz)];
                if (g >= 0 && conflicts(tx, ty, g)) cmask |= 1u << t;
            }
        }
        cmask = __reduce_or_sync(0xffffffffu, cmask);
        // resolve in try order (every lane the same decisions)
        unsigned amask = 0u;
        int nacc = 0;
        for (int t = 0; t < K; ++t) {
            const double tx = __shfl_sync(0xffffffffu, px, t), ty = __shfl_sync(0xffffffffu, py, t);
            const int tgx = __shfl_sync(0xffffffffu, gx, t), tgy = __shfl_sync(0xffffffffu, gy, t);
            const int tin = __shfl_sync(0xffffffffu, inb, t);
            bool ok = tin && !((cmask >> t) & 1u);
            for (int u = 0; u < t; ++u) {
                const double ux = __shfl_sync(0xffffffffu, px, u), uy = __shfl_sync(0xffffffffu, py, u);
                const int ucell = __shfl_sync(0xffffffffu, gx, u) + __shfl_sync(0xffffffffu, gy, u) * gw;
                if (!ok || !((amask >> u) & 1u)) continue;
                // is u's cell among the 25 that try t checks (flat indices (xx + yy gw) mod gsz,
                // xx in [tgx-2, tgx+2])? per row yy: (ucell - yy gw - (tgx-2)) mod gsz <= 4
                bool seen = false;
                for (int b = 0; b < 5 && !seen; ++b) seen = pymod(ucell - (tgy - 2 + b) * gw - (tgx - 2), gsz) <= 4;
                if (seen) {
                    double dx = fabs(tx - ux), dy = fabs(ty - uy);
                    if (dx > width * 0.5) dx -= width;
                    if (dy > height * 0.5) dy -= height;
                    if ((dx * dx + dy * dy) <= rSq) ok = false;
                }
            }
            if (!ok) continue;
            if (npts + nacc >= S.gsz) { overflow = true; break; }
            amask |= 1u << t;
            ++nacc;
        }
        if (lane < K && ((amask >> lane) & 1u)) {
            const int rank = __popc(amask & below);
            const int id = npts + rank;
            M.ptx[id] = px; M.pty[id] = py;
            M.queue[nq + rank] = id;
            M.grid[gx + gy * gw] = id;
        }
        __syncwarp();
        npts += nacc;
        nq += nacc;
    }
    if (overflow && lane == 0) *status |= HS_ST_POISSON_OVERFLOW;
    __syncwarp();
    // keep points with x < max(r, w - r), y < max(r, h - r) (PBC=True default), then offset;
    // in grid-cell order, compacted by the warp
    const double lx = fmax(r, width - r), ly = fmax(r, height - r);
    const double ox = (double)(int)(rnd_at(call) * width), oy = (double)(int)(rnd_at(call + 1) * height);
    call += 2;
    int k = 0;
    for (int g0 = 0; g0 < gsz; g0 += 32) {
        const int g = g0 + lane;
        const int p = g < gsz ? M.grid[g] : -1;
        bool keep = false;
        int ix = 0, iy = 0;
        if (p >= 0) {
            const double x = M.ptx[p], y = M.pty[p];
            keep = x >= 0.0 && y >= 0.0 && x < lx && y < ly;
            if (keep) {
                const double fx = fmod(x + ox, width), fy = fmod(y + oy, height);
                // nearest cell index, ties to the lower index
                ix = (int)floor(fx); if (fx - ix > 0.5) ix += 1; ix = min(max(ix, 0), L.nx - 1);
                iy = (int)floor(fy); if (fy - iy > 0.5) iy += 1; iy = min(max(iy, 0), L.ny - 1);
            }
        }
        const unsigned b = __ballot_sync(0xffffffffu, keep);
        const int pos = k + __popc(b & below);
        if (keep && pos < S.cap) { S.py[pos] = iy; S.px[pos] = ix; }
        k += __popc(b);
    }
    if (k > S.cap) { if (lane == 0) *status |= HS_ST_POISSON_OVERFLOW; k = S.cap; }
    __syncwarp();
    return k;
}

// Block-wide exclusive scans of two flags at once (3 barriers in total).
HS_DEV void block_excl_scan2(int f0, int f1, int *wt, int &pre0, int &pre1, int &tot0, int &tot1) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const unsigned b0 = __ballot_sync(0xffffffffu, f0), b1 = __ballot_sync(0xffffffffu, f1);
    if (lane == 0) { wt[warp] = __popc(b0); wt[33 + warp] = __popc(b1); }
    __syncthreads();
    if (warp == 0) {
        int v0 = lane < nw ? wt[lane] : 0, v1 = lane < nw ? wt[33 + lane] : 0;
        int i0 = v0, i1 = v1;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int a = __shfl_up_sync(0xffffffffu, i0, o), b = __shfl_up_sync(0xffffffffu, i1, o);
            if (lane >= o) { i0 += a; i1 += b; }
        }
        if (lane < nw) { wt[lane] = i0 - v0; wt[33 + lane] = i1 - v1; }
        if (lane == 31) { wt[32] = i0; wt[65] = i1; }
    }
    __syncthreads();
    const unsigned below = (1u << lane) - 1u;
    pre0 = wt[warp] + __popc(b0 & below);
    pre1 = wt[33 + warp] + __popc(b1 & below);
    tot0 = wt[32]; tot1 = wt[65];
    __syncthreads();
}

// Grid-selection Metropolis step with one candidate per thread (n_sc <= blockDim.x), kept in
// registers: the supercell filter, the offset and the occupation filter of
// hotspice/core.py:534-553 and 484-487 become one pair of fused ballot scans. Returns false,
// without side effects, when the step needs the rare branches (no candidate survives the
// supercell filter -> _select_single, or none is occupied -> select() retries); the general
// path then runs the step from the same RNG call.
HS_DEV bool metro_grid_fast(const HsLattice &L, HsCounters *C, const HsSwitchList &sw, const HsGridPlan &P,
                            uint64_t call) {
    __shared__ int wt[66];
    __shared__ int s_bins[256];
    __shared__ double s_tsum[32];
    const int t = threadIdx.x;
    int ox, oy;
    if (L.pbc) {
        ox = (int)floor(hs_u53(L.seed, call, 0u) * L.nx);
        oy = (int)floor(hs_u53(L.seed, call + 1, 0u) * L.ny);
    } else {
        ox = -P.Rx + (int)floor(hs_u53(L.seed, call, 0u) * (2.0 * P.Rx));
        oy = -P.Ry + (int)floor(hs_u53(L.seed, call + 1, 0u) * (2.0 * P.Ry));
    }
    if (P.Rx == L.nx) ox = 0;
    if (P.Ry == L.ny) oy = 0;
    const int phase = pymod(oy, L.uy) * L.ux + pymod(ox, L.ux);
    const int off = P.phase_off[phase], len = P.phase_off[phase + 1] - off;
    if (len <= 0) return false;
    const int nscx = (min(P.snx, L.nx) + 1) / 2;
    int ok = 0, valid = 0, x = 0, y = 0;
    if (t < P.n_sc) {
        const int pick = (int)floor(hs_u53(L.seed, call + 2, (uint32_t)t) * len);
        const int yx = __ldg(P.phase_yx + off + pick);
        x = 2 * (t % nscx) * P.Rx + (yx & 0xffff);
        y = 2 * (t / nscx) * P.Ry + (yx >> 16);
        if (L.pbc) {
            ok = x < max(P.Rx, L.nx - P.Rx) && y < max(P.Ry, L.ny - P.Ry);
            x = (x + ox) % L.nx; y = (y + oy) % L.ny;
        } else {
            x += ox; y += oy;
            ok = x >= 0 && x < L.nx && y >= 0 && y < L.ny;
        }
        valid = ok && L.occ[(int64_t)y * L.nx + x] != 0;
    }
    int pre_ok, r, n_ok, k;
    block_excl_scan2(ok, valid, wt, pre_ok, r, n_ok, k);
    if (n_ok == 0 || k == 0) return false;  // block-uniform
    const bool mtime = P.metropolis_time != 0;
    const uint64_t call_time = call + 3;
    const uint64_t call_acc = mtime ? call + 4 : call + 3;
    for (int b = t; b < 256; b += blockDim.x) s_bins[b] = 0;
    int acc = 0;
    double tpart = 0.0;
    long long near = 0;
    int8_t m_old = 0;
    float mm_old = 0.f;
    if (valid) {
        const int64_t i = (int64_t)y * L.nx + x;
        // the spin and moment for the flip are loaded with the energies (one round trip)
        m_old = __ldcg(L.m + i);
        mm_old = __ldcg(L.mm + i);
        double E, Ep;
        hs_energy_at(L, y, x, E, Ep);
        const double beta = hs_beta(L, i);
        const double p = fmin(fmax(exp(2.0 * E * beta), 1e-10), 1e10);
        if (mtime) {
            double b1, b2;
            hs_barriers(L, y, x, b1, b2);
            const double u = hs_u53(L.seed, call_time, (uint32_t)r);
            tpart = -log(u) / P.attempt_freq / (double)L.n_occ * exp(fmin(b1, b2) * beta);
        }
        const double u = hs_u53(L.seed, call_acc, (uint32_t)r);
        acc = u < p;
        if (fabs(u - p) <= p * beta * 2e-6 * fabs(E) && p < 1e10 && p > 1e-10) near = 1;
    }
    int pa, dummy, nacc, dtot;
    block_excl_scan2(acc, 0, wt, pa, dummy, nacc, dtot);
    const int bin = acc ? (x % L.ux) + (y % L.uy) * L.ux : 0;
    if (acc) {
        const int64_t i = (int64_t)y * L.nx + x;
        L.m[i] = (int8_t)(-m_old);
        L.mm[i] = -mm_old;
        if (pa < sw.cap) { sw.y[pa] = y; sw.x[pa] = x; }
        atomicAdd(&s_bins[bin], 1);
    }
    if (mtime) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) tpart += __shfl_xor_sync(0xffffffffu, tpart, o);
        if ((t & 31) == 0) s_tsum[t >> 5] = tpart;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) near += __shfl_xor_sync(0xffffffffu, near, o);
    if ((t & 31) == 0 && near) atomicAdd((unsigned long long *)&C->near_threshold, (unsigned long long)near);
    __syncthreads();
    if (acc && sw.mode && pa < sw.cap) sw.mode[pa] = s_bins[bin] > L.trunc_cutoff ? 1 : 0;
    if (t == 0) {
        if (mtime) {
            double ts = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) ts += s_tsum[w];
            C->t += ts;
        }
        const int ncap = min(nacc, sw.cap);
        C->attempted += k;
        C->switches += ncap;
        C->rng_call = call_acc + 1;
        C->n_sw = ncap;
        C->steps += 1;
        if (nacc > sw.cap) C->status |= HS_ST_SWITCH_OVERFLOW;
    }
    __syncthreads();
    return true;
}

// The same step as metro_grid_fast when every supercell fits one warp (n_sc <= 32), executed
// by a single warp with ballots instead of block scans: candidates, acceptances and switch
// list in the same order, the per-sublattice switch counts by __match_any_sync, the
// METROPOLIS_TIME sum by the same xor-shuffle tree (the other warps held only zeros), so the
// results are identical. Returns false, without side effects, when the step needs the rare
// branches (the general path then runs it from the same call).
HS_DEV bool metro_grid_warp(const HsLattice &L, HsCounters *C, const HsSwitchList &sw, const HsGridPlan &P,
                            uint64_t call) {
    const int lane = threadIdx.x & 31;
    // the lane's pick variate does not depend on the offsets: drawn alongside them
    const double upick = lane < P.n_sc ? hs_u53(L.seed, call + 2, (uint32_t)lane) : 0.0;
    int ox, oy;
    if (L.pbc) {
        ox = (int)floor(hs_u53(L.seed, call, 0u) * L.nx);
        oy = (int)floor(hs_u53(L.seed, call + 1, 0u) * L.ny);
    } else {
        ox = -P.Rx + (int)floor(hs_u53(L.seed, call, 0u) * (2.0 * P.Rx));
        oy = -P.Ry + (int)floor(hs_u53(L.seed, call + 1, 0u) * (2.0 * P.Ry));
    }
    if (P.Rx == L.nx) ox = 0;
    if (P.Ry == L.ny) oy = 0;
    const int phase = pymod(oy, L.uy) * L.ux + pymod(ox, L.ux);
    const int off = P.phase_off[phase], len = P.phase_off[phase + 1] - off;
    if (len <= 0) return false;
    const int nscx = (min(P.snx, L.nx) + 1) / 2;
    int ok = 0, valid = 0, x = 0, y = 0;
    if (lane < P.n_sc) {
        const int pick = (int)floor(upick * len);
        const int yx = __ldg(P.phase_yx + off + pick);
        x = 2 * (lane % nscx) * P.Rx + (yx & 0xffff);
        y = 2 * (lane / nscx) * P.Ry + (yx >> 16);
        if (L.pbc) {
            ok = x < max(P.Rx, L.nx - P.Rx) && y < max(P.Ry, L.ny - P.Ry);
            x = (x + ox) % L.nx; y = (y + oy) % L.ny;
        } else {
            x += ox; y += oy;
            ok = x >= 0 && x < L.nx && y >= 0 && y < L.ny;
        }
        valid = ok && __ldg(L.occ + (int64_t)y * L.nx + x) != 0;
    }
    const unsigned below = (1u << lane) - 1u;
    const unsigned okb = __ballot_sync(0xffffffffu, ok), vb = __ballot_sync(0xffffffffu, valid);
    const int k = __popc(vb);
    if (okb == 0u || k == 0) return false;   // warp-uniform
    const int r = __popc(vb & below);
    const bool mtime = P.metropolis_time != 0;
    const uint64_t call_time = call + 3;
    const uint64_t call_acc = mtime ? call + 4 : call + 3;
    int acc = 0;
    double tpart = 0.0;
    int near = 0;
    int8_t m_old = 0;
    float mm_old = 0.f;
    if (valid) {
        const int64_t i = (int64_t)y * L.nx + x;
        // the spin and moment for the flip are loaded with the energies (one round trip)
        m_old = __ldcg(L.m + i);
        mm_old = __ldcg(L.mm + i);
        double E, Ep;
        hs_energy_at(L, y, x, E, Ep);
        const double beta = hs_beta(L, i);
        const double p = fmin(fmax(exp(2.0 * E * beta), 1e-10), 1e10);
        if (mtime) {
            double b1, b2;
            hs_barriers(L, y, x, b1, b2);
            const double u = hs_u53(L.seed, call_time, (uint32_t)r);
            tpart = -log(u) / P.attempt_freq / (double)L.n_occ * exp(fmin(b1, b2) * beta);
        }
        const double u = hs_u53(L.seed, call_acc, (uint32_t)r);
        acc = u < p;
        if (fabs(u - p) <= p * beta * 2e-6 * fabs(E) && p < 1e10 && p > 1e-10) near = 1;
    }
    const unsigned accb = __ballot_sync(0xffffffffu, acc);
    const int nacc = __popc(accb), pa = __popc(accb & below);
    const int bin = (x % L.ux) + (y % L.uy) * L.ux;
    const unsigned same = __match_any_sync(0xffffffffu, acc ? bin : -1);
    if (acc) {
        const int64_t i = (int64_t)y * L.nx + x;
        L.m[i] = (int8_t)(-m_old);
        L.mm[i] = -mm_old;
        if (pa < sw.cap) {
            sw.y[pa] = y; sw.x[pa] = x;
            if (sw.mode) sw.mode[pa] = __popc(same & accb) > L.trunc_cutoff ? 1 : 0;
        }
    }
    if (mtime) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) tpart += __shfl_xor_sync(0xffffffffu, tpart, o);
    }
    const int nnear = __popc(__ballot_sync(0xffffffffu, near));
    if (lane == 0) {
        if (nnear) C->near_threshold += nnear;
        if (mtime) C->t += tpart;
        const int ncap = min(nacc, sw.cap);
        C->attempted += k;
        C->switches += ncap;
        C->rng_call = call_acc + 1;
        C->n_sw = ncap;
        C->steps += 1;
        if (nacc > sw.cap) C->status |= HS_ST_SWITCH_OVERFLOW;
    }
    return true;
}

// One Metropolis step executed by one CTA (selection, acceptance, flips, switch list).
HS_DEV void metro_step_cta(const HsLattice &L, HsCounters *C, const HsSwitchList &sw, const HsGridPlan &P,
                           const MetroScratch &S, void *ws = nullptr, int ws_bytes = 0) {
    __shared__ int warp_tot[33];
    __shared__ int s_k;
    __shared__ uint64_t s_call;
    __shared__ int s_status;
    __shared__ int s_bins[256];
    __shared__ double s_tsum[32];
    if (C->done) return;
    if (!hs_progress_continue(C, L.n_occ)) {
        if (threadIdx.x == 0) { C->done = 1; C->n_sw = 0; }
        return;
    }
    uint64_t call = C->rng_call;
    if (P.sample_scheme == HS_SAMPLE_GRID && P.n_sc <= 32) {
        __shared__ int s_done;
        if (threadIdx.x < 32) {
            const bool d = metro_grid_warp(L, C, sw, P, call);
            if (threadIdx.x == 0) s_done = d;
        }
        __syncthreads();
        const int d = s_done;
        __syncthreads();   // s_done is rewritten by the next step
        if (d) return;
    } else if (P.sample_scheme == HS_SAMPLE_GRID && P.n_sc <= (int)blockDim.x && L.ux * L.uy <= 256 &&
               metro_grid_fast(L, C, sw, P, call))
        return;
    if (threadIdx.x == 0) s_status = 0;
    int k = 0;
    int retry = 0;
    for (; retry < MAX_RETRY; ++retry) {
        // ---- selection -------------------------------------------------------------------
        if (P.sample_scheme == HS_SAMPLE_GRID) {
            int ox, oy;
            if (L.pbc) {
                ox = (int)floor(hs_u53(L.seed, call, 0u) * L.nx);
                oy = (int)floor(hs_u53(L.seed, call + 1, 0u) * L.ny);
            } else {
                ox = -P.Rx + (int)floor(hs_u53(L.seed, call, 0u) * (2.0 * P.Rx));
                oy = -P.Ry + (int)floor(hs_u53(L.seed, call + 1, 0u) * (2.0 * P.Ry));
            }
            if (P.Rx == L.nx) ox = 0;
            if (P.Ry == L.ny) oy = 0;
            const int phase = pymod(oy, L.uy) * L.ux + pymod(ox, L.ux);
            const int off = P.phase_off[phase], len = P.phase_off[phase + 1] - off;
            const int nscx = (min(P.snx, L.nx) + 1) / 2;
            const int limx = max(P.Rx, L.nx - P.Rx), limy = max(P.Ry, L.ny - P.Ry);
            // candidates, in the row-major supercell order of ixx[:sny:2, :snx:2].ravel()
            for (int t = threadIdx.x; t < P.n_sc; t += blockDim.x) {
                int ix = -1, iy = -1;
                if (len > 0) {
                    const int pick = (int)floor(hs_u53(L.seed, call + 2, (uint32_t)t) * len);
                    const int yx = P.phase_yx[off + pick];
                    ix = 2 * (t % nscx) * P.Rx + (yx & 0xffff);
                    iy = 2 * (t / nscx) * P.Ry + (yx >> 16);
                }
                S.py[t] = iy; S.px[t] = ix;
            }
            if (len <= 0 && threadIdx.x == 0) s_status |= HS_ST_SELECT_RETRY;
            __syncthreads();
            const int nx = L.nx, ny = L.ny, pbc = L.pbc;
            k = block_compact(S.py, S.px, P.n_sc, [&](int y, int x) {
                if (x < 0) return false;
                if (pbc) return x < limx && y < limy;
                x += ox; y += oy;
                return x >= 0 && x < nx && y >= 0 && y < ny;
            }, warp_tot);
            for (int t = threadIdx.x; t < k; t += blockDim.x) {
                if (pbc) { S.px[t] = (S.px[t] + ox) % L.nx; S.py[t] = (S.py[t] + oy) % L.ny; }
                else { S.px[t] += ox; S.py[t] += oy; }
            }
            call += 3;
            __syncthreads();
            if (k == 0) {  // no sample survived: _select_single (core.py:558)
                const int i = (int)floor(hs_u53(L.seed, call, 0u) * L.n_occ);
                if (threadIdx.x == 0) { const int f = L.nonzero[i]; S.py[0] = f / L.nx; S.px[0] = f % L.nx; }
                call += 1;
                k = 1;
            }
        } else if (P.sample_scheme == HS_SAMPLE_SINGLE) {
            const int i = (int)floor(hs_u53(L.seed, call, 0u) * L.n_occ);
            if (threadIdx.x == 0) { const int f = L.nonzero[i]; S.py[0] = f / L.nx; S.px[0] = f % L.nx; }
            call += 1;
            k = 1;
        } else {  // Poisson
            if (threadIdx.x < 32) {
                uint64_t c = call;
                int st = 0;
                // the sampler's arrays in the shared workspace when they fit, else in the scratch
                const int64_t g = (int64_t)hs_poisson_grid_cells(L, P);
                PoissonMem M;
                if (ws && hs_poisson_mem_bytes(g) <= ws_bytes) M = poisson_mem_in(ws, (int)g);
                else { M.grid = S.grid; M.ptx = S.ptx; M.pty = S.pty; M.queue = S.queue; }
                const int n = poisson_warp(L, P, S, M, c, &st);
                if (threadIdx.x == 0) { s_k = n; s_call = c; s_status |= st; }
            }
            __syncthreads();
            k = s_k;
            call = s_call;
        }
        __syncthreads();
        // ---- select(): drop unoccupied picks, retry if none is left (core.py:484-487) -------
        const int8_t *occ = L.occ;
        const int nx = L.nx;
        k = block_compact(S.py, S.px, k, [&](int y, int x) { return occ[(int64_t)y * nx + x] != 0; }, warp_tot);
        if (k > 0) break;
    }
    if (retry == MAX_RETRY) {
        if (threadIdx.x == 0) { C->status |= HS_ST_SELECT_RETRY; C->rng_call = call; C->n_sw = 0; }
        return;
    }
    // ---- acceptance --------------------------------------------------------------------------
    const bool mtime = P.metropolis_time != 0;
    const uint64_t call_time = call;
    const uint64_t call_acc = mtime ? call + 1 : call;
    for (int b = threadIdx.x; b < 256; b += blockDim.x) s_bins[b] = 0;
    double tpart = 0.0;
    long long near = 0;
    int acc_base = 0;
    __syncthreads();
    for (int base = 0; base < k; base += blockDim.x) {
        const int t = base + threadIdx.x;
        int acc = 0, y = 0, x = 0;
        if (t < k) {
            y = S.py[t]; x = S.px[t];
            const int64_t i = (int64_t)y * L.nx + x;
            double E, Ep;
            hs_energy_at(L, y, x, E, Ep);
            const double dE = -2.0 * E;
            const double beta = hs_beta(L, i);
            const double p = fmin(fmax(exp(-dE * beta), 1e-10), 1e10);
            if (mtime) {
                double b1, b2;
                hs_barriers(L, y, x, b1, b2);
                const double u = hs_u53(L.seed, call_time, (uint32_t)t);
                tpart += -log(u) / P.attempt_freq / (double)L.n_occ * exp(fmin(b1, b2) * beta);
            }
            const double u = hs_u53(L.seed, call_acc, (uint32_t)t);
            acc = u < p;
            // decision margin below a 1e-6 relative energy perturbation
            if (fabs(u - p) <= p * beta * 2e-6 * fabs(E) && p < 1e10 && p > 1e-10) near += 1;
        }
        int tot;
        const int pre = block_excl_scan(acc, warp_tot, tot);
        if (acc) {
            const int out = acc_base + pre;
            if (out < sw.cap) { sw.y[out] = y; sw.x[out] = x; }
        }
        acc_base += tot;
    }
    const int nacc = acc_base;
    // time sum (METROPOLIS_TIME)
    if (mtime) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) tpart += __shfl_xor_sync(0xffffffffu, tpart, o);
        if ((threadIdx.x & 31) == 0) s_tsum[threadIdx.x >> 5] = tpart;
    }
    // near-threshold count
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) near += __shfl_xor_sync(0xffffffffu, near, o);
    if ((threadIdx.x & 31) == 0 && near) atomicAdd((unsigned long long *)&C->near_threshold, (unsigned long long)near);
    __syncthreads();
    const int ncap = min(nacc, sw.cap);
    // flips and per-sublattice counts
    for (int t = threadIdx.x; t < ncap; t += blockDim.x) {
        const int y = sw.y[t], x = sw.x[t];
        const int64_t i = (int64_t)y * L.nx + x;
        L.m[i] = (int8_t)(-L.m[i]);
        L.mm[i] = -L.mm[i];
        const int bin = (x % L.ux) + (y % L.uy) * L.ux;
        if (bin < 256) atomicAdd(&s_bins[bin], 1);
    }
    __syncthreads();
    if (sw.mode)
        for (int t = threadIdx.x; t < ncap; t += blockDim.x) {
            const int y = sw.y[t], x = sw.x[t];
            const int bin = (x % L.ux) + (y % L.uy) * L.ux;
            sw.mode[t] = (bin < 256 && s_bins[bin] > L.trunc_cutoff) ? 1 : 0;
        }
    if (threadIdx.x == 0) {
        if (mtime) {
            double ts = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) ts += s_tsum[w];
            C->t += ts;
        }
        C->attempted += k;
        C->switches += ncap;
        C->rng_call = call_acc + 1;
        C->n_sw = ncap;
        C->steps += 1;
        C->status |= s_status;
        if (nacc > sw.cap) C->status |= HS_ST_SWITCH_OVERFLOW;
    }
}

// ---- Wolff -------------------------------------------------------------------------------

constexpr int WT = 1024;

struct WolffScratch {
    int32_t *chk_ep;   // epoch in which the cell was checked (seed or frontier)
    int32_t *cl_ep;    // epoch in which the cell joined the cluster
    int32_t *cl_layer; // layer in which it joined
    int32_t *list;     // cluster cells in BFS order (capacity N)
    int32_t *cand;     // frontier of the current layer (capacity N)
    int32_t *epoch;    // last epoch used with these stamps; kept here, not in the counters, so that
                       // restoring an earlier counter state never makes an old stamp current again
};

// One Wolff cluster step executed by one CTA.
HS_DEV void wolff_step_cta(const HsLattice &L, HsCounters *C, const HsSwitchList &sw, const WolffScratch &S) {
    __shared__ int s_ncand, s_nacc, s_epoch;
    if (C->done) return;
    if (!hs_progress_continue(C, L.n_occ)) {
        if (threadIdx.x == 0) { C->done = 1; C->n_sw = 0; }
        return;
    }
    const int nx = L.nx, ny = L.ny;
    const int64_t N = (int64_t)nx * ny;
    uint64_t call = C->rng_call;
    if (threadIdx.x == 0) { s_epoch = *S.epoch + 1; *S.epoch = s_epoch; C->epoch = s_epoch; }
    // seed: _select_single (np.random.randint(n) -> nonzero index)
    const int seed = L.nonzero[(int)floor(hs_u53(L.seed, call, 0u) * L.n_occ)];
    call += 1;
    __syncthreads();
    const int epoch = s_epoch;
    const int8_t ms = L.m[seed];
    if (threadIdx.x == 0) {
        S.chk_ep[seed] = epoch;
        S.cl_ep[seed] = epoch;
        S.cl_layer[seed] = 0;
        S.list[0] = seed;
    }
    int lstart = 0, lend = 1;
    const int ch = L.nn_h / 2, cw = L.nn_w / 2;
    const double m2J = -2.0 * L.J;
    int layer = 1;
    for (; layer <= (int)N + 1; ++layer) {
        if (threadIdx.x == 0) { s_ncand = 0; s_nacc = 0; }
        __syncthreads();
        // frontier: unchecked same-spin cells j with q = j + c - b for a new cell q, mask[b] != 0
        for (int t = lstart + threadIdx.x; t < lend; t += blockDim.x) {
            const int q = S.list[t];
            const int qy = q / nx, qx = q % nx;
            for (int a = 0; a < L.nn_h; ++a)
                for (int b = 0; b < L.nn_w; ++b) {
                    if (!L.nn[a * L.nn_w + b]) continue;
                    int jy = qy - ch + a, jx = qx - cw + b;
                    if (L.pbc) { jy = hs_wrap(jy, ny); jx = hs_wrap(jx, nx); }
                    else if (jy < 0 || jy >= ny || jx < 0 || jx >= nx) continue;
                    const int j = jy * nx + jx;
                    if (L.m[j] != ms) continue;
                    if (atomicExch(&S.chk_ep[j], epoch) == epoch) continue;
                    S.cand[atomicAdd(&s_ncand, 1)] = j;
                }
        }
        __syncthreads();
        const int ncand = s_ncand;
        if (ncand == 0) break;  // empty frontier: the reference's while-loop ends, no draw
        for (int t = threadIdx.x; t < ncand; t += blockDim.x) {
            const int j = S.cand[t];
            const int jy = j / nx, jx = j % nx;
            int count = 0;
            for (int a = 0; a < L.nn_h; ++a)
                for (int b = 0; b < L.nn_w; ++b) {
                    const int w = L.nn[a * L.nn_w + b];
                    if (!w) continue;
                    int yy = jy + ch - a, xx = jx + cw - b;
                    if (L.pbc) { yy = hs_wrap(yy, ny); xx = hs_wrap(xx, nx); }
                    else if (yy < 0 || yy >= ny || xx < 0 || xx >= nx) continue;
                    const int k = yy * nx + xx;
                    if (S.cl_ep[k] == epoch && S.cl_layer[k] < layer) count += w;
                }
            // bond = 1 - exp(-2 J / kBT * count), kBT = 1/beta (hotspice/core.py:599)
            double bond;
            if (L.wolff_bond && count <= 24) {
                bond = L.wolff_bond[count];
            } else {
                const double kBT = 1.0 / hs_beta(L, j);
                bond = 1.0 - exp(m2J / kBT * (double)count);
            }
            const double u = hs_u53(L.seed, call, (uint32_t)j);
            if (!(u > bond)) {
                S.cl_ep[j] = epoch;
                S.cl_layer[j] = layer;
                S.list[lend + atomicAdd(&s_nacc, 1)] = j;
            }
        }
        call += 1;
        __syncthreads();
        lstart = lend;
        lend += s_nacc;
    }
    if (layer > (int)N + 1 && threadIdx.x == 0) C->status |= HS_ST_WOLFF_OVERFLOW;
    // flip the cluster; counters as in core.py:714-716
    for (int t = threadIdx.x; t < lend; t += blockDim.x) {
        const int j = S.list[t];
        L.m[j] = (int8_t)(-L.m[j]);
        L.mm[j] = -L.mm[j];
        if (t < sw.cap) { sw.y[t] = j / nx; sw.x[t] = j % nx; if (sw.mode) sw.mode[t] = 0; }
    }
    if (threadIdx.x == 0) {
        C->attempted += lend;
        C->switches += lend;
        C->rng_call = call;
        C->n_sw = min(lend, sw.cap);
        C->steps += 1;
        if (lend > sw.cap) C->status |= HS_ST_SWITCH_OVERFLOW;
    }
}

// ---- Néel -------------------------------------------------------------------------------
// Final stage of a Néel step once the global argmin `w` of the log-domain keys is known:
// switching time in FP64, flip, counters and the one-entry switch list
// (hotspice/core.py:699-709). Executed by a single thread.
// The flip a Néel decision made, for a caller that writes it itself (neel_finalize's `defer`).
struct NeelFlip { int64_t i; int y, x; int8_t m_new; float mm_new; bool flip; };
HS_DEV void neel_apply(const HsLattice &L, const HsSwitchList &sw, const NeelFlip &f) {
    L.m[f.i] = f.m_new;
    L.mm[f.i] = f.mm_new;
    sw.y[0] = f.y;
    sw.x[0] = f.x;
    if (sw.mode) sw.mode[0] = 0;
}

// `defer`: the flip (spin, moment, switch list) is returned there instead of being written.
HS_DEV void neel_finalize(const HsLattice &L, HsCounters *C, const HsSwitchList &sw, HsKeyIdx w, uint64_t call,
                          double bmin, bool unif, bool two, double attempt_freq, NeelFlip *defer = nullptr) {
    if (defer) defer->flip = false;
    C->rng_call = call + 1;
    C->attempted += 1;
    C->steps += 1;
    const double t_eff = C->progress ? (C->t_max - (C->t - C->t0)) : C->t_max;
    if (w.idx < 0) {  // no occupied cell: nanargmin would raise; record and stop
        C->status |= HS_ST_SELECT_RETRY;
        C->n_sw = 0;
        C->t += t_eff;
        return;
    }
    const int64_t i = w.idx;
    // the cell's spin and moment: carried by the scan's record, else loaded first, so that
    // their round trips overlap the switching-time arithmetic below
    const int8_t m_old = w.m ? (int8_t)w.m : L.m[i];
    const float mm_old = w.m ? w.mm : L.mm[i];
    const int y = (int)(i / L.nx), x = (int)(i % L.nx);
    // the barriers the scan computed for this cell (the same operations as hs_barriers)
    const double b1 = w.b1, b2 = w.b2;
    const double beta = hs_beta(L, i);
    const double e1 = hs_exp1_f64(hs_u53(L.seed, call, (uint32_t)i));
    double time;
    if (!two) {
        // time = E1 * exp((b - bmin) beta) * exp(bmin beta) / nu   (hotspice/core.py:698-700)
        time = unif ? e1 * exp(b1 * beta) / attempt_freq
                    : e1 * exp((b1 - bmin) * beta) * exp(bmin * beta) / attempt_freq;
    } else {
        const double bm = fmin(b1, b2), dd = fabs(b1 - b2);
        // tau = E1 / (exp(-(b1-bmin) beta) + exp(-(b2-bmin) beta)); nu halves (core.py:691-693)
        const double scale = exp((bm - bmin) * beta) / (1.0 + exp(-dd * beta));
        time = e1 * scale * exp(bmin * beta) / (attempt_freq / 2.0);
    }
    C->last_time = time;
    if (time > t_eff || isnan(time)) {
        C->t += t_eff;
        C->n_sw = 0;
        return;
    }
    const NeelFlip f{i, y, x, (int8_t)(-m_old), -mm_old, true};
    if (defer) *defer = f;
    else neel_apply(L, sw, f);
    C->switches += 1;
    C->t += time;
    C->n_sw = 1;
}

// Scratch layout of the Metropolis step (shared by the host launcher and the engine).
HS_HD inline int64_t hs_align_up_d(int64_t v, int64_t a) { return (v + a - 1) / a * a; }
HS_HD inline void hs_metro_sizes(const HsLattice &L, const HsGridPlan &P, int &cap, int &gsz) {
    cap = P.n_sc > 1 ? P.n_sc : 1;
    gsz = 0;
    if (P.sample_scheme == HS_SAMPLE_POISSON) {
        const double g = hs_poisson_grid_cells(L, P);
        gsz = g <= (double)HS_POISSON_GRID_MAX ? (int)g : HS_POISSON_GRID_MAX;   // validated by the entry points
        cap = cap > gsz ? cap : gsz;
    }
}

// Barriers of hotspice/core.py:625-656 from an already-loaded total energy E, perpendicular
// energy Ep (before m_perp_factor) and E_B.
HS_DEV void hs_barriers_from(const HsLattice &L, double E, double Ep, double EB, double &b1, double &b2) {
    const double dE = -2.0 * E;
    const double Ecur = -dE / 2.0;
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

// Néel log-domain keys (see hs_neel.cu) of the occupied cells, folded into `best`. The work
// is the occupied cells start, start + stride, ... : taken from the occupied-cell list when the
// lattice is sparse (fewer than 3/4 of its cells hold a magnet), else all cells with an
// occupation test. The loads of NEEL_UNR cells are issued before any of them is used, so that
// one thread keeps several L2 round trips in flight. A cell whose key cannot beat the thread's
// best so far is skipped before the accurate logarithms: log E1 >= log u (E1 = -log(1 - u) >= u)
// and the two-channel term is >= -ln 2, so log u + (b_low - b_min) beta - ln 2 (less a margin
// for the fast logarithm) is a lower bound of the key. The (key, index) minimum does not depend
// on the visiting order or on the skipping (ties go to the smaller index; only cells whose key
// is strictly larger than a key already seen are skipped).
// Néel barrier cache (engine only): per cell s = b_low * beta (uniform beta), rounded down to
// float, +inf for an empty cell. It lives in the Néel scratch at this offset and is valid only
// inside one engine launch (built by the launch's first step, refreshed by the window update).
constexpr int64_t HS_NEEL_CACHE_OFFSET = 65536;
HS_DEV float neel_cache_value(const HsLattice &L, double E, double Ep, double EB) {
    double b1, b2;
    hs_barriers_from(L, E, Ep, EB, b1, b2);
    return __double2float_rd(fmin(b1, b2) * L.beta_uniform);
}

#ifndef HS_NEEL_UNROLL
#define HS_NEEL_UNROLL 3
#endif
constexpr int NEEL_UNR = HS_NEEL_UNROLL;
HS_DEV HsKeyIdx neel_scan_range(const HsLattice &L, int64_t start64, int64_t stride64, int64_t N64, uint64_t call,
                                double bmin, HsKeyIdx best, float *cache = nullptr) {
    const bool two = L.use_perp != 0;
    const bool sparse = 4 * (int64_t)L.n_occ < 3 * N64;
    const int M = sparse ? L.n_occ : (int)N64;     // cell indices fit in int (HsKeyIdx.idx)
    const int start = (int)start64, stride = (int)stride64;
    const double slack = (two ? 0.6931471805599453 : 0.0) + 1e-4;
    for (int base = start; base < M; base += stride * NEEL_UNR) {
        int ci[NEEL_UNR];
        int8_t oc[NEEL_UNR], mv[NEEL_UNR];
        double ed[NEEL_UNR], edp[NEEL_UNR];
        float zf[NEEL_UNR], zfp[NEEL_UNR], eb[NEEL_UNR], bt[NEEL_UNR];
#pragma unroll
        for (int k = 0; k < NEEL_UNR; ++k) {
            const int j = base + k * stride;
            const bool v = j < M;
            ci[k] = v ? (sparse ? __ldg(L.nonzero + j) : j) : 0;
        }
#pragma unroll
        for (int k = 0; k < NEEL_UNR; ++k) {
            const bool v = base + k * stride < M;
            const int i = ci[k];
            oc[k] = v ? (sparse ? (int8_t)1 : L.occ[i]) : (int8_t)0;
            mv[k] = v ? __ldcg(L.m + i) : (int8_t)0;
            ed[k] = (v && L.has_dipolar) ? __ldcg(L.E_dip + i) : 0.0;
            edp[k] = (v && L.has_dipolar && two) ? __ldcg(L.E_dip_perp + i) : 0.0;
            zf[k] = (v && L.zee) ? __ldg(L.zee + i) : 0.f;
            zfp[k] = (v && L.zee && two) ? __ldg(L.zee_perp + i) : 0.f;
            eb[k] = v ? __ldg(L.E_B + i) : 0.f;
            bt[k] = (v && L.beta_uniform <= 0.0) ? __ldg(L.beta + i) : 0.f;
        }
        // branch-free phases, so the NEEL_UNR Philox chains and barrier evaluations interleave
        double u[NEEL_UNR], lb[NEEL_UNR], b1v[NEEL_UNR], b2v[NEEL_UNR], btv[NEEL_UNR];
#pragma unroll
        for (int k = 0; k < NEEL_UNR; ++k) u[k] = hs_u53(L.seed, call, (uint32_t)ci[k]);
#pragma unroll
        for (int k = 0; k < NEEL_UNR; ++k) {
            double E = ed[k], Ep = edp[k];
            if (L.zee) { E += (double)mv[k] * (double)zf[k]; if (two) Ep += (double)mv[k] * (double)zfp[k]; }
            if (L.has_exchange) {
                double e, ep;
                hs_exchange_at(L, ci[k] / L.nx, ci[k] % L.nx, e, ep);
                E += e;
                if (two) Ep += ep;
            }
            hs_barriers_from(L, E, Ep, (double)eb[k], b1v[k], b2v[k]);
            btv[k] = L.beta_uniform > 0.0 ? L.beta_uniform : (double)bt[k];
            const double bm = two ? fmin(b1v[k], b2v[k]) : b1v[k];
            lb[k] = (double)__logf((float)u[k]) + (bm - bmin) * btv[k] - slack;
            if (cache && base + k * stride < M) cache[ci[k]] = oc[k] ? __double2float_rd(bm * btv[k]) : INFINITY;
        }
#pragma unroll
        for (int k = 0; k < NEEL_UNR; ++k) {
            if (!oc[k]) continue;
            if (best.idx >= 0 && lb[k] > best.key) continue;
            const double b1 = b1v[k], b2 = b2v[k], beta = btv[k];
            const double le1 = (double)hs_log_exp1_f32(u[k]);
            double key;
            if (!two) key = le1 + (b1 - bmin) * beta;
            else {
                const double bm = fmin(b1, b2), dd = fabs(b1 - b2);
                key = le1 + (bm - bmin) * beta - (double)log1pf(expf((float)(-dd * beta)));
            }
            best = hs_kmin(best, HsKeyIdx{key, ci[k], b1, b2});
        }
    }
    return best;
}

// Exact log-domain key of occupied cell i from its energies (uniform beta, b_min = 0): the
// operations of neel_scan_range, so both give the same key bit for bit.
HS_DEV HsKeyIdx neel_key_exact(const HsLattice &L, int i, uint32_t call_lo, uint32_t call_hi, const HsRoundKeys &RK) {
    const bool two = L.use_perp != 0;
    const double beta = L.beta_uniform;
    const double uk = hs_u53_of(hs_philox_rk((uint32_t)i, call_lo, call_hi, 0u, RK));
    double E = L.has_dipolar ? __ldcg(L.E_dip + i) : 0.0;
    double Ep = (L.has_dipolar && two) ? __ldcg(L.E_dip_perp + i) : 0.0;
    const int mv = __ldcg(L.m + i);
    const float mm = __ldcg(L.mm + i);   // carried to the decision (same round trip)
    if (L.zee) { E += (double)mv * (double)__ldg(L.zee + i); if (two) Ep += (double)mv * (double)__ldg(L.zee_perp + i); }
    double b1, b2;
    hs_barriers_from(L, E, Ep, (double)__ldg(L.E_B + i), b1, b2);
    const double le1 = (double)hs_log_exp1_f32(uk);
    double key;
    if (!two) key = le1 + b1 * beta;
    else {
        const double bm = fmin(b1, b2), dd = fabs(b1 - b2);
        key = le1 + bm * beta - (double)log1pf(expf((float)(-dd * beta)));
    }
    return HsKeyIdx{key, i, b1, b2, mm, mv};
}

// Per-warp queue of the cached scan (shared memory, ints): cells whose lower bound does not rule
// them out wait there and are evaluated 32 at a time, one per lane.
constexpr int NEEL_QCAP = 64;

// An upper bound of the exact key of a cell (neel_key_exact) from its first Philox word and its
// cached s = b_low beta rounded down: u53 < u24 + 2^-24 and E1 = -log1p(-u) grows with u, the
// two-channel term only lowers the key, s is below the next float up; 1e-4 covers the float
// rounding of the logarithms (their absolute errors here are below 1e-5).
HS_DEV double neel_key_upper(HsU4 w, float s) {
    const float uh = hs_u24_low(w) + 5.9604644775390625e-08f;   // exact: a multiple of 2^-24 <= 1
    const float le = __logf(-log1pf(-uh));
    const double sh = (double)s + fabs((double)s) * 2.4e-7 + 1e-30;
    return (double)le + sh + 1e-4;
}

// The same scan from the barrier cache (uniform beta, b_min = 0): per cell the cached
// s = b_low beta, the Philox variate and the lower bound log u + s; the exact key (computed as
// in neel_scan_range, from the energies) only for the cells the bound does not rule out.
// Warp-collective: the 32 lanes of a warp call it together with consecutive `start`s
// (start = warp base + lane). The warp keeps T, an upper bound of the smallest key among the
// cells it has seen (the minimum of the cells' upper bounds, neel_key_upper, and of the exact
// keys found), and admits a cell only when its lower bound is not above T. Admitted cells go to
// the warp's queue `q` (NEEL_QCAP ints) in ballot order and are evaluated exactly when 32 or
// more wait, with every lane busy: a per-lane branch to the exact evaluation would cost the warp
// that evaluation on almost every cell, since some lane of 32 usually admits one. The cell of
// the smallest key always has its lower bound below T (every upper bound is at least that key),
// so every cell that can win or tie is evaluated, and the (key, index) minimum is that of the
// exhaustive scan. Returns the warp's minimum on every lane.
HS_DEV HsKeyIdx neel_scan_cached(const HsLattice &L, const float *cache, int64_t start64, int64_t stride64, int64_t N64,
                                 uint64_t call, HsKeyIdx best, int *q) {
    const bool two = L.use_perp != 0;
    const bool sparse = 4 * (int64_t)L.n_occ < 3 * N64;
    const int M = sparse ? L.n_occ : (int)N64;
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    const int start0 = (int)start64 - lane, stride = (int)stride64;
    const double slack = (two ? 0.6931471805599453 : 0.0) + 1e-4;
    const HsRoundKeys RK = hs_round_keys(L.seed);
    const uint32_t call_lo = (uint32_t)call, call_hi = (uint32_t)(call >> 32);
    if (__any_sync(0xffffffffu, best.idx >= 0)) best = hs_warp_kmin(best);
    double T = best.idx >= 0 ? best.key : INFINITY;   // warp-uniform
    int qn = 0;                                       // warp-uniform
    auto flush = [&]() {
        __syncwarp();
        for (int b = 0; b < qn; b += 32) {
            HsKeyIdx c{0.0, -1};
            if (b + lane < qn) c = neel_key_exact(L, q[b + lane], call_lo, call_hi, RK);
            best = hs_kmin(best, hs_warp_kmin(c));
        }
        if (best.idx >= 0) T = fmin(T, best.key);
        qn = 0;
        __syncwarp();
    };
    // cell indices and cached bounds of the chunk at `base` (cells beyond M: index 0, bound +inf)
    auto load = [&](int base, int *c, float *b) {
#pragma unroll
        for (int k = 0; k < NEEL_UNR; ++k) {
            const int j = base + lane + k * stride;
            c[k] = j < M ? (sparse ? __ldg(L.nonzero + j) : j) : 0;
        }
#pragma unroll
        for (int k = 0; k < NEEL_UNR; ++k) b[k] = base + lane + k * stride < M ? __ldcg(cache + c[k]) : INFINITY;
    };
    int ci[NEEL_UNR];
    float sc[NEEL_UNR];
    load(start0, ci, sc);
    for (int base = start0; base < M; base += stride * NEEL_UNR) {   // warp-uniform trip count
        // the next chunk's loads are issued first and complete while this chunk computes
        int cn[NEEL_UNR];
        float sn[NEEL_UNR];
        load(base + stride * NEEL_UNR, cn, sn);
        HsU4 wv[NEEL_UNR];
#pragma unroll
        for (int k = 0; k < NEEL_UNR; ++k) wv[k] = hs_philox_rk((uint32_t)ci[k], call_lo, call_hi, 0u, RK);
        // bounds from the first Philox word (below u53): the FP64 variate only for admitted cells
        double lbk[NEEL_UNR];
        double lmin = INFINITY;   // the lane's smallest bound of the chunk, with its word and s
        HsU4 wmin = wv[0];
        float smin = sc[0];
#pragma unroll
        for (int k = 0; k < NEEL_UNR; ++k) {
            lbk[k] = sc[k] != INFINITY ? (double)__logf(hs_u24_low(wv[k])) + (double)sc[k] - slack : INFINITY;
            if (lbk[k] < lmin) { lmin = lbk[k]; wmin = wv[k]; smin = sc[k]; }
        }
        if (__any_sync(0xffffffffu, lmin <= T)) {
            // lower T with the upper bound of each lane's best cell of the chunk (warp-uniform)
            double t = lmin <= T ? fmin(T, neel_key_upper(wmin, smin)) : T;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) t = fmin(t, __shfl_xor_sync(0xffffffffu, t, o));
            T = t;
        }
#pragma unroll
        for (int k = 0; k < NEEL_UNR; ++k) {
            const bool adm = sc[k] != INFINITY && lbk[k] <= T;
            const unsigned m = __ballot_sync(0xffffffffu, adm);
            if (m) {
                if (adm) q[qn + __popc(m & below)] = ci[k];
                qn += __popc(m);
                if (qn >= 32) flush();
            }
        }
#pragma unroll
        for (int k = 0; k < NEEL_UNR; ++k) { ci[k] = cn[k]; sc[k] = sn[k]; }
    }
    if (qn) flush();
    return best;
}
