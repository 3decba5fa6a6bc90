// (a) incremental dipolar energy update and (b, checker) direct full recompute.
//
// The incremental update is a deterministic gather: the lattice is cut into tiles of
// 16 rows x (32*VEC) columns (8 warps, 2 rows each), every CTA keeps the switches whose
// window reaches its tile (in their original order, so the summation order never depends on
// scheduling; all warps scan the list together, 1024 switches per round), and each thread
// owns VEC consecutive cells of 2 rows: it reads E and mm once (float4 when the row is
// 16-byte aligned), accumulates sum_s mm_s * K_s(j - s) over the switches, and writes E
// back once. Semantics follow hotspice/energies.py:310-366:
//   HS_UPDATE_SINGLE   E_j += 2 pref mm_j acc_j; then E_s = -E_s          (update_single)
//   HS_UPDATE_MULTIPLE E_s = -E_s for every switch; E_j += 2 pref mm_j acc_j (update_multiple)
// E_perp follows E, except that with L.dip_keep_perp_sign a list of more than one switch
// leaves E_perp_s unnegated (DiMonopolarEnergy.update_multiple, hotspice/energies.py:718-719).
// A switch in "truncated" mode (more than SIMULTANEOUS_SWITCHES_CONVOLUTION_OR_SUM_CUTOFF
// switches on its sublattice, hotspice/energies.py:343-353) contributes only the
// (2k+1)^2 crop of its kernel with wrap (PBC) or zero fill, like convolve2d(..., 'same').
#include "hs_common.cuh"
#include "hs_internal.h"

#include "hs_steps.cuh"

namespace {

// Tile shape and occupancy of the incremental update (compile-time; the defaults are the
// measured best on B200 for the benchmarked windows).
#ifndef HS_UPD_WARPS
#define HS_UPD_WARPS 8
#endif
#ifndef HS_UPD_RPW
#define HS_UPD_RPW 2
#endif
#ifndef HS_UPD_MIN_CTAS
#define HS_UPD_MIN_CTAS 4
#endif
#ifndef HS_UPD_SCAN
#define HS_UPD_SCAN 2
#endif
#ifndef HS_UPD_PERSIST_MIN_TILES
#define HS_UPD_PERSIST_MIN_TILES 296   // two tiles per SM of a B200 (148 SMs)
#endif
constexpr int UPD_WARPS = HS_UPD_WARPS;            // warps per CTA
constexpr int UPD_RPW = HS_UPD_RPW;                // rows per warp
constexpr int UPD_TY = UPD_WARPS * UPD_RPW;        // rows per tile
constexpr int UPD_SCAN = HS_UPD_SCAN;              // switches per lane per staging round
constexpr int UPD_ROUND = UPD_WARPS * 32 * UPD_SCAN;
constexpr int UPD_LOC = 2048;                      // staged switches per pass

template <int VEC>
__global__ void __launch_bounds__(32 * UPD_WARPS, HS_UPD_MIN_CTAS)
dip_update_kernel(HsLattice L, HsSwitchList sw, const int32_t *n_sw_dev, int n_host, int semantics,
                  const HsCounters *C) {
    if (C && C->done) return;
    const int nsw = n_sw_dev ? *n_sw_dev : n_host;
    if (nsw <= 0) return;
    constexpr int TX = 32 * VEC;
    const int tiles_x = (L.nx + TX - 1) / TX;
    const int ty0 = (blockIdx.x / tiles_x) * UPD_TY;
    const int tx0 = (blockIdx.x % tiles_x) * TX;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int x0 = tx0 + lane * VEC;

    __shared__ SwInfo s_sw[UPD_LOC];
    __shared__ int s_cnt[UPD_WARPS];
    float acc[UPD_RPW][VEC], accp[UPD_RPW][VEC];
    unsigned touched = 0u, negate = 0u;   // bit r * VEC + v
#pragma unroll
    for (int r = 0; r < UPD_RPW; ++r)
#pragma unroll
        for (int v = 0; v < VEC; ++v) { acc[r][v] = 0.f; accp[r][v] = 0.f; }

    const float pref2 = (float)(2.0 * L.dip_pref);
    // a one-switch update is update_single in the reference (hotspice/core.py:250-253)
    const bool flip_perp = !(L.dip_keep_perp_sign && nsw > 1);
    const bool vec_rows = VEC == 4 && x0 + 3 < L.nx && (L.nx & 3) == 0;
    for (int base = 0; base < nsw;) {
        // Stage, in list order, the switches of [base, ...) whose window reaches this tile. All
        // warps scan: warp w takes the block [s + w 32 UPD_SCAN, ...) of each round, its hits are
        // compacted in order behind those of the warps before it.
        int n = 0, s = base;
        while (s < nsw && n + UPD_ROUND <= UPD_LOC) {
            int ky[UPD_SCAN], kx[UPD_SCAN], kmode[UPD_SCAN];
            bool val[UPD_SCAN];
#pragma unroll
            for (int u = 0; u < UPD_SCAN; ++u) {
                const int k = s + (warp * UPD_SCAN + u) * 32 + lane;
                val[u] = k < nsw;
                ky[u] = val[u] ? sw.y[k] : 0;
                kx[u] = val[u] ? sw.x[k] : 0;
                kmode[u] = (val[u] && sw.mode) ? sw.mode[k] : 0;
            }
            SwInfo w[UPD_SCAN];
            bool hit[UPD_SCAN];
#pragma unroll
            for (int u = 0; u < UPD_SCAN; ++u) {
                w[u] = SwInfo{ky[u], kx[u], kmode[u], -1, 0.f};
                hit[u] = false;
                if (!val[u]) continue;
                w[u].sub = hs_sub(L, ky[u], kx[u]);
                if (w[u].sub >= 0) {
                    int hy, wy_, hx, wx_;
                    hs_window(L, kmode[u], true, hy, wy_);
                    hs_window(L, kmode[u], false, hx, wx_);
                    hit[u] = hs_axis_overlap(ky[u], hy, wy_, L.ny, ty0, UPD_TY) &&
                             hs_axis_overlap(kx[u], hx, wx_, L.nx, tx0, TX);
                } else {
                    // no kernel for this unit-cell site: only the sign flip of E applies
                    hit[u] = semantics == HS_UPDATE_MULTIPLE && ky[u] >= ty0 && ky[u] < ty0 + UPD_TY &&
                             kx[u] >= tx0 && kx[u] < tx0 + TX;
                }
            }
#pragma unroll
            for (int u = 0; u < UPD_SCAN; ++u)
                if (hit[u] && w[u].sub >= 0) w[u].mm = L.mm[(int64_t)ky[u] * L.nx + kx[u]];
            unsigned bal[UPD_SCAN];
            int wc = 0;
#pragma unroll
            for (int u = 0; u < UPD_SCAN; ++u) { bal[u] = __ballot_sync(0xffffffffu, hit[u]); wc += __popc(bal[u]); }
            if (lane == 0) s_cnt[warp] = wc;
            __syncthreads();
            int off = n, tot = n;
#pragma unroll
            for (int q = 0; q < UPD_WARPS; ++q) { if (q < warp) off += s_cnt[q]; tot += s_cnt[q]; }
            const unsigned below = (1u << lane) - 1u;
#pragma unroll
            for (int u = 0; u < UPD_SCAN; ++u) {
                if (hit[u]) s_sw[off + __popc(bal[u] & below)] = w[u];
                off += __popc(bal[u]);
            }
            __syncthreads();
            n = tot;
            s += UPD_ROUND;
        }
        const int KW = 2 * L.dip_wx + 1, KH = 2 * L.dip_wy + 1;
        for (int q = 0; q < n; ++q) {
            const SwInfo w = s_sw[q];
            if (w.sub >= 0 && !w.mode && !L.dip_wrap) {
                // exact window without wrapping: one kernel row per target row, consecutive
                // columns across the lanes (the same values hs_contrib would add)
                const int64_t kb = (int64_t)w.sub * KH * KW + (L.dip_wx - w.x);
#pragma unroll
                for (int r = 0; r < UPD_RPW; ++r) {
                    const int y = ty0 + warp * UPD_RPW + r;
                    if (y >= L.ny) continue;
                    const int dy = y - w.y;
                    const bool rowin = dy >= -L.dip_wy && dy <= L.dip_wy;
                    const float *Kr = L.K + kb + (int64_t)(dy + L.dip_wy) * KW;
                    const float *Kpr = L.use_perp ? L.Kpo + kb + (int64_t)(dy + L.dip_wy) * KW : nullptr;
#pragma unroll
                    for (int v = 0; v < VEC; ++v) {
                        const int x = x0 + v;
                        if (x >= L.nx) continue;
                        touched |= 1u << (r * VEC + v);
                        const int dx = x - w.x;
                        if (rowin && dx >= -L.dip_wx && dx <= L.dip_wx) {
                            acc[r][v] += w.mm * __ldg(Kr + x);
                            if (L.use_perp) accp[r][v] += w.mm * __ldg(Kpr + x);
                            if (dy == 0 && dx == 0) negate |= 1u << (r * VEC + v);
                        }
                    }
                }
                continue;
            }
#pragma unroll
            for (int r = 0; r < UPD_RPW; ++r) {
                const int y = ty0 + warp * UPD_RPW + r;
                if (y >= L.ny) continue;
#pragma unroll
                for (int v = 0; v < VEC; ++v) {
                    const int x = x0 + v;
                    if (x >= L.nx) continue;
                    if (w.sub >= 0) {
                        float a = acc[r][v], ap = accp[r][v];
                        hs_contrib(L, w, y, x, a, ap);
                        acc[r][v] = a; accp[r][v] = ap;
                    }
                    touched |= 1u << (r * VEC + v);
                    if (w.y == y && w.x == x) negate |= 1u << (r * VEC + v);
                }
            }
        }
        __syncthreads();
        base = s;
    }
#pragma unroll
    for (int r = 0; r < UPD_RPW; ++r) {
        const int y = ty0 + warp * UPD_RPW + r;
        if (y >= L.ny) continue;
        const int64_t row = (int64_t)y * L.nx;
        if (vec_rows) {
            if (!((touched >> (r * VEC)) & 0xFu)) continue;
            const float4 mm4 = *reinterpret_cast<const float4 *>(L.mm + row + x0);
            const float mmv[4] = {mm4.x, mm4.y, mm4.z, mm4.w};
            const double2 e01 = *reinterpret_cast<const double2 *>(L.E_dip + row + x0);
            const double2 e23 = *reinterpret_cast<const double2 *>(L.E_dip + row + x0 + 2);
            double ev[4] = {e01.x, e01.y, e23.x, e23.y};
            double pv[4] = {0.0, 0.0, 0.0, 0.0};
            if (L.use_perp) {
                const double2 p01 = *reinterpret_cast<const double2 *>(L.E_dip_perp + row + x0);
                const double2 p23 = *reinterpret_cast<const double2 *>(L.E_dip_perp + row + x0 + 2);
                pv[0] = p01.x; pv[1] = p01.y; pv[2] = p23.x; pv[3] = p23.y;
            }
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                const bool ng = (negate >> (r * VEC + v)) & 1u;
                if (semantics == HS_UPDATE_MULTIPLE) {
                    if (ng) { ev[v] = -ev[v]; if (flip_perp) pv[v] = -pv[v]; }
                    ev[v] += (double)(pref2 * (mmv[v] * acc[r][v]));
                    pv[v] += (double)(pref2 * (mmv[v] * accp[r][v]));
                } else {
                    ev[v] += (double)(pref2 * (mmv[v] * acc[r][v]));
                    pv[v] += (double)(pref2 * (mmv[v] * accp[r][v]));
                    if (ng) { ev[v] = -ev[v]; pv[v] = -pv[v]; }
                }
            }
            *reinterpret_cast<double2 *>(L.E_dip + row + x0) = make_double2(ev[0], ev[1]);
            *reinterpret_cast<double2 *>(L.E_dip + row + x0 + 2) = make_double2(ev[2], ev[3]);
            if (L.use_perp) {
                *reinterpret_cast<double2 *>(L.E_dip_perp + row + x0) = make_double2(pv[0], pv[1]);
                *reinterpret_cast<double2 *>(L.E_dip_perp + row + x0 + 2) = make_double2(pv[2], pv[3]);
            }
            continue;
        }
#pragma unroll
        for (int v = 0; v < VEC; ++v) {
            const int x = x0 + v;
            if (x >= L.nx || !((touched >> (r * VEC + v)) & 1u)) continue;
            const bool ng = (negate >> (r * VEC + v)) & 1u;
            const float mmv = L.mm[row + x];
            double e = L.E_dip[row + x];
            if (semantics == HS_UPDATE_MULTIPLE) { if (ng) e = -e; e += (double)(pref2 * (mmv * acc[r][v])); }
            else { e += (double)(pref2 * (mmv * acc[r][v])); if (ng) e = -e; }
            L.E_dip[row + x] = e;
            if (L.use_perp) {
                double p = L.E_dip_perp[row + x];
                if (semantics == HS_UPDATE_MULTIPLE) { if (ng && flip_perp) p = -p; p += (double)(pref2 * (mmv * accp[r][v])); }
                else { p += (double)(pref2 * (mmv * accp[r][v])); if (ng) p = -p; }
                L.E_dip_perp[row + x] = p;
            }
        }
    }
}

// Persistent form of dip_update_kernel for lists of at most UPD_PLOC switches. A CTA stages the
// whole list in dynamic shared memory once, then walks tiles (tile = blockIdx.x, + gridDim.x,
// ...). For every tile the CTA builds the list of switches that reach it, in list order (each
// thread tests a contiguous chunk of the list; one block scan places the hits), and it builds
// the NEXT tile's list and prefetches that tile's rows of E, E_perp and m*moment into L2 while it
// processes the current one.
// Per cell the arithmetic and the summation order are those of dip_update_kernel, so both give
// the same bits.
constexpr int UPD_PLOC = 4096;

struct PersistSmem {                // layout of the dynamic shared memory (n = list bound)
    SwInfo *sw;                     // [n] the staged list
    int16_t *hit[2];                // [n] each: hit lists of the current and the next tile
    static int64_t bytes(int n) { return (int64_t)n * sizeof(SwInfo) + 2 * hs_align_up_d(2LL * n, 16) + 64; }
};

template <int VEC>
__global__ void __launch_bounds__(32 * UPD_WARPS, HS_UPD_MIN_CTAS)
dip_update_persist_kernel(HsLattice L, HsSwitchList sw, const int32_t *n_sw_dev, int n_host, int semantics,
                          const HsCounters *C, int tiles, int cap) {
    if (C && C->done) return;
    const int nsw = n_sw_dev ? *n_sw_dev : n_host;
    if (nsw <= 0 || nsw > cap) return;   // the launcher sends longer lists to dip_update_kernel
    constexpr int TX = 32 * VEC;
    extern __shared__ __align__(16) unsigned char s_dyn[];
    SwInfo *s_sw = reinterpret_cast<SwInfo *>(s_dyn);
    int16_t *s_hit[2];
    s_hit[0] = reinterpret_cast<int16_t *>(s_dyn + (int64_t)cap * sizeof(SwInfo));
    s_hit[1] = s_hit[0] + hs_align_up_d(cap, 8);
    __shared__ int s_tot[UPD_WARPS + 1];
    __shared__ int s_nhit[2];
    {   // stage the list; the loads of 8 entries per thread are issued before any is used
        constexpr int SU = 8;
        for (int k0 = threadIdx.x; k0 < nsw; k0 += SU * blockDim.x) {
            int yy[SU], xx[SU], md[SU], sb[SU];
            float mv[SU];
#pragma unroll
            for (int j = 0; j < SU; ++j) {
                const int k = k0 + j * blockDim.x;
                const bool v = k < nsw;
                yy[j] = v ? sw.y[k] : 0;
                xx[j] = v ? sw.x[k] : 0;
                md[j] = (v && sw.mode) ? sw.mode[k] : 0;
            }
#pragma unroll
            for (int j = 0; j < SU; ++j) {
                sb[j] = k0 + j * blockDim.x < nsw ? hs_sub(L, yy[j], xx[j]) : -1;
                mv[j] = sb[j] >= 0 ? L.mm[(int64_t)yy[j] * L.nx + xx[j]] : 0.f;
            }
#pragma unroll
            for (int j = 0; j < SU; ++j)
                if (k0 + j * blockDim.x < nsw) s_sw[k0 + j * blockDim.x] = SwInfo{yy[j], xx[j], md[j], sb[j], mv[j]};
        }
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int tiles_x = (L.nx + TX - 1) / TX;
    const float pref2 = (float)(2.0 * L.dip_pref);
    const bool flip_perp = !(L.dip_keep_perp_sign && nsw > 1);
    const int KW = 2 * L.dip_wx + 1, KH = 2 * L.dip_wy + 1;
    const int chunk = (nsw + blockDim.x - 1) / blockDim.x;   // switches tested by each thread

    // does switch w reach (or, without a kernel, sit in) the tile at (ty0, tx0)?
    auto hits_tile = [&](const SwInfo &w, int ty0, int tx0) {
        if (w.sub < 0)
            return semantics == HS_UPDATE_MULTIPLE && w.y >= ty0 && w.y < ty0 + UPD_TY && w.x >= tx0 && w.x < tx0 + TX;
        int hy, wy_, hx, wx_;
        hs_window(L, w.mode, true, hy, wy_);
        hs_window(L, w.mode, false, hx, wx_);
        return hs_axis_overlap(w.y, hy, wy_, L.ny, ty0, UPD_TY) && hs_axis_overlap(w.x, hx, wx_, L.nx, tx0, TX);
    };

    // the hits of `tile` in list order into s_hit[b], their count into s_nhit[b] (block-wide:
    // every thread must call it)
    auto build_hits = [&](int tile, int b) {
        const int ty0 = (tile / tiles_x) * UPD_TY, tx0 = (tile % tiles_x) * TX;
        const int k0 = min(nsw, (int)threadIdx.x * chunk), k1 = min(nsw, k0 + chunk);
        unsigned mask = 0u;   // chunk <= 16 (UPD_PLOC / blockDim.x)
        int cnt = 0;
        for (int k = k0; k < k1; ++k)
            if (hits_tile(s_sw[k], ty0, tx0)) { mask |= 1u << (k - k0); ++cnt; }
        // exclusive block scan of the per-thread counts
        int incl = cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) { const int t = __shfl_up_sync(0xffffffffu, incl, o); if (lane >= o) incl += t; }
        if (lane == 31) s_tot[warp] = incl;
        __syncthreads();
        if (threadIdx.x == 0) {
            int acc = 0;
            for (int q = 0; q < UPD_WARPS; ++q) { const int v = s_tot[q]; s_tot[q] = acc; acc += v; }
            s_nhit[b] = acc;
        }
        __syncthreads();
        int pos = s_tot[warp] + incl - cnt;
        for (int k = k0; mask; ++k, mask >>= 1)
            if (mask & 1u) s_hit[b][pos++] = (int16_t)k;
        if (s_nhit[b] > 0) {   // block-uniform: prefetch this warp's rows of the tile into L2
            for (int r = 0; r < UPD_RPW; ++r) {
                const int y = ty0 + warp * UPD_RPW + r, x = tx0 + lane * VEC;
                if (y < L.ny && x < L.nx) {
                    const int64_t i = (int64_t)y * L.nx + x;
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(L.E_dip + i));
                    asm volatile("prefetch.global.L2 [%0];" ::"l"(L.mm + i));
                    if (L.use_perp) asm volatile("prefetch.global.L2 [%0];" ::"l"(L.E_dip_perp + i));
                }
            }
        }
    };

    int tile = blockIdx.x, cur = 0;
    if (tile < tiles) build_hits(tile, cur);
    __syncthreads();
    for (; tile < tiles; tile += gridDim.x, cur ^= 1) {
        const int next = tile + gridDim.x;
        if (next < tiles) build_hits(next, cur ^ 1);   // the next tile's list and its rows' prefetch
        const int nhit = s_nhit[cur];
        const int16_t *hl = s_hit[cur];
        const int y0 = (tile / tiles_x) * UPD_TY + warp * UPD_RPW;
        const int tx0 = (tile % tiles_x) * TX;
        const int x0 = tx0 + lane * VEC;
        if (nhit > 0 && y0 < L.ny) {
            const int nrows = min(UPD_RPW, L.ny - y0);
            float acc[UPD_RPW][VEC], accp[UPD_RPW][VEC];
#pragma unroll
            for (int r = 0; r < UPD_RPW; ++r)
#pragma unroll
                for (int v = 0; v < VEC; ++v) { acc[r][v] = 0.f; accp[r][v] = 0.f; }
            unsigned touched = 0u, negate = 0u;   // bit r * VEC + v
            auto apply = [&](const SwInfo &w) {
                if (w.sub >= 0 && !w.mode && !L.dip_wrap) {
                    const int64_t kb = (int64_t)w.sub * KH * KW + (L.dip_wx - w.x);
                    // every VEC cells of the lane inside the window's columns (the common case
                    // for windows wider than a lane): no per-cell column tests
                    const bool inner = x0 >= w.x - L.dip_wx && x0 + VEC - 1 <= w.x + L.dip_wx && x0 + VEC - 1 < L.nx;
#pragma unroll
                    for (int r = 0; r < UPD_RPW; ++r) {
                        if (r >= nrows) continue;
                        const int y = y0 + r;
                        const int dy = y - w.y;
                        const bool rowin = dy >= -L.dip_wy && dy <= L.dip_wy;
                        const float *Kr = L.K + kb + (int64_t)(dy + L.dip_wy) * KW;
                        const float *Kpr = L.use_perp ? L.Kpo + kb + (int64_t)(dy + L.dip_wy) * KW : nullptr;
                        if (inner) {
                            touched |= ((1u << VEC) - 1u) << (r * VEC);
                            if (!rowin) continue;
                            float kv[VEC], kp[VEC];
#pragma unroll
                            for (int v = 0; v < VEC; ++v) kv[v] = __ldg(Kr + x0 + v);
                            if (L.use_perp) {
#pragma unroll
                                for (int v = 0; v < VEC; ++v) kp[v] = __ldg(Kpr + x0 + v);
                            }
#pragma unroll
                            for (int v = 0; v < VEC; ++v) {
                                acc[r][v] += w.mm * kv[v];
                                if (L.use_perp) accp[r][v] += w.mm * kp[v];
                            }
                            const int ds = w.x - x0;
                            if (dy == 0 && ds >= 0 && ds < VEC) negate |= 1u << (r * VEC + ds);
                            continue;
                        }
#pragma unroll
                        for (int v = 0; v < VEC; ++v) {
                            const int x = x0 + v;
                            if (x >= L.nx) continue;
                            touched |= 1u << (r * VEC + v);
                            const int dx = x - w.x;
                            if (rowin && dx >= -L.dip_wx && dx <= L.dip_wx) {
                                acc[r][v] += w.mm * __ldg(Kr + x);
                                if (L.use_perp) accp[r][v] += w.mm * __ldg(Kpr + x);
                                if (dy == 0 && dx == 0) negate |= 1u << (r * VEC + v);
                            }
                        }
                    }
                    return;
                }
#pragma unroll
                for (int r = 0; r < UPD_RPW; ++r) {
                    if (r >= nrows) continue;
                    const int y = y0 + r;
#pragma unroll
                    for (int v = 0; v < VEC; ++v) {
                        const int x = x0 + v;
                        if (x >= L.nx) continue;
                        if (w.sub >= 0) {
                            float a = acc[r][v], ap = accp[r][v];
                            hs_contrib(L, w, y, x, a, ap);
                            acc[r][v] = a; accp[r][v] = ap;
                        }
                        touched |= 1u << (r * VEC + v);
                        if (w.y == y && w.x == x) negate |= 1u << (r * VEC + v);
                    }
                }
            };
            if (nhit <= 64) {
                // Each lane applies only the hits whose window reaches its own cells (a mask over
                // the tile's list, visited in list order): with windows narrower than the tile,
                // most hits of a tile miss most lanes, and skipping them changes no sum.
                unsigned long long mine = 0ull;
                const int yhi = y0 + nrows - 1, xhi = x0 + VEC - 1;
                for (int h = 0; h < nhit; ++h) {
                    const SwInfo w = s_sw[hl[h]];
                    const bool exact = w.sub >= 0 && !w.mode && !L.dip_wrap;
                    const bool reach = !exact || (w.y - L.dip_wy <= yhi && w.y + L.dip_wy >= y0 &&
                                                  w.x - L.dip_wx <= xhi && w.x + L.dip_wx >= x0);
                    if (reach) mine |= 1ull << h;
                }
                for (; mine; mine &= mine - 1ull) apply(s_sw[hl[__ffsll((long long)mine) - 1]]);
            } else {
                for (int h = 0; h < nhit; ++h) apply(s_sw[hl[h]]);
            }
            const bool vec_rows = VEC == 4 && x0 + 3 < L.nx && (L.nx & 3) == 0;
#pragma unroll
            for (int r = 0; r < UPD_RPW; ++r) {
                if (r >= nrows) continue;
                const int64_t row = (int64_t)(y0 + r) * L.nx;
                if (vec_rows) {
                    if (!((touched >> (r * VEC)) & 0xFu)) continue;
                    const float4 mm4 = *reinterpret_cast<const float4 *>(L.mm + row + x0);
                    const float mmv[4] = {mm4.x, mm4.y, mm4.z, mm4.w};
                    const double2 e01 = *reinterpret_cast<const double2 *>(L.E_dip + row + x0);
                    const double2 e23 = *reinterpret_cast<const double2 *>(L.E_dip + row + x0 + 2);
                    double ev[4] = {e01.x, e01.y, e23.x, e23.y};
                    double pv[4] = {0.0, 0.0, 0.0, 0.0};
                    if (L.use_perp) {
                        const double2 p01 = *reinterpret_cast<const double2 *>(L.E_dip_perp + row + x0);
                        const double2 p23 = *reinterpret_cast<const double2 *>(L.E_dip_perp + row + x0 + 2);
                        pv[0] = p01.x; pv[1] = p01.y; pv[2] = p23.x; pv[3] = p23.y;
                    }
#pragma unroll
                    for (int v = 0; v < 4; ++v) {
                        const bool ng = (negate >> (r * VEC + v)) & 1u;
                        if (semantics == HS_UPDATE_MULTIPLE) {
                            if (ng) { ev[v] = -ev[v]; if (flip_perp) pv[v] = -pv[v]; }
                            ev[v] += (double)(pref2 * (mmv[v] * acc[r][v]));
                            pv[v] += (double)(pref2 * (mmv[v] * accp[r][v]));
                        } else {
                            ev[v] += (double)(pref2 * (mmv[v] * acc[r][v]));
                            pv[v] += (double)(pref2 * (mmv[v] * accp[r][v]));
                            if (ng) { ev[v] = -ev[v]; pv[v] = -pv[v]; }
                        }
                    }
                    *reinterpret_cast<double2 *>(L.E_dip + row + x0) = make_double2(ev[0], ev[1]);
                    *reinterpret_cast<double2 *>(L.E_dip + row + x0 + 2) = make_double2(ev[2], ev[3]);
                    if (L.use_perp) {
                        *reinterpret_cast<double2 *>(L.E_dip_perp + row + x0) = make_double2(pv[0], pv[1]);
                        *reinterpret_cast<double2 *>(L.E_dip_perp + row + x0 + 2) = make_double2(pv[2], pv[3]);
                    }
                    continue;
                }
#pragma unroll
                for (int v = 0; v < VEC; ++v) {
                    const int x = x0 + v;
                    if (x >= L.nx || !((touched >> (r * VEC + v)) & 1u)) continue;
                    const bool ng = (negate >> (r * VEC + v)) & 1u;
                    const float mmv = L.mm[row + x];
                    double e = L.E_dip[row + x];
                    if (semantics == HS_UPDATE_MULTIPLE) { if (ng) e = -e; e += (double)(pref2 * (mmv * acc[r][v])); }
                    else { e += (double)(pref2 * (mmv * acc[r][v])); if (ng) e = -e; }
                    L.E_dip[row + x] = e;
                    if (L.use_perp) {
                        double p = L.E_dip_perp[row + x];
                        if (semantics == HS_UPDATE_MULTIPLE) { if (ng && flip_perp) p = -p; p += (double)(pref2 * (mmv * accp[r][v])); }
                        else { p += (double)(pref2 * (mmv * accp[r][v])); if (ng) p = -p; }
                        L.E_dip_perp[row + x] = p;
                    }
                }
            }
        }
        __syncthreads();   // s_hit[cur] is rebuilt two tiles on; s_nhit[cur ^ 1] is read next
    }
}

// Direct-sum full recompute, one thread per target cell (hotspice/energies.py:290-308):
//   E_i = pref * mu_i * m_i * sum_j K_{s(i)}(j - i) * mm_j,  E_perp with the perp-self kernel.
template <typename Acc, bool FULLWIN>
__global__ void dip_full_direct_kernel(HsLattice L, int fp64, double *E64, double *Ep64) {
    const int64_t N = (int64_t)L.nx * L.ny;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        const int y = (int)(i / L.nx), x = (int)(i % L.nx);
        const int s = hs_sub(L, y, x);
        const int mi = L.m[i];
        Acc acc = 0, accp = 0;
        if (s >= 0 && mi != 0) {
            if (FULLWIN) {
                for (int jy = 0; jy < L.ny; ++jy) {
                    const int dy = jy - y;
                    const int64_t jrow = (int64_t)jy * L.nx;
                    for (int jx = 0; jx < L.nx; ++jx) {
                        const Acc mj = (Acc)L.mm[jrow + jx];
                        if (mj == (Acc)0) continue;
                        acc += (Acc)hs_kval(L, L.K, s, dy, jx - x) * mj;
                        if (L.use_perp) accp += (Acc)hs_kval(L, L.Kps, s, dy, jx - x) * mj;
                    }
                }
            } else {
                for (int dy = -L.dip_wy; dy <= L.dip_wy; ++dy) {
                    int jy = y + dy;
                    if (L.dip_wrap) jy = hs_wrap(jy, L.ny);
                    else if (jy < 0 || jy >= L.ny) continue;
                    const int64_t jrow = (int64_t)jy * L.nx;
                    for (int dx = -L.dip_wx; dx <= L.dip_wx; ++dx) {
                        int jx = x + dx;
                        if (L.dip_wrap) jx = hs_wrap(jx, L.nx);
                        else if (jx < 0 || jx >= L.nx) continue;
                        const Acc mj = (Acc)L.mm[jrow + jx];
                        if (mj == (Acc)0) continue;
                        const int64_t k = (int64_t)s * (2 * L.dip_wy + 1) * (2 * L.dip_wx + 1) +
                                          (int64_t)(dy + L.dip_wy) * (2 * L.dip_wx + 1) + (dx + L.dip_wx);
                        acc += (Acc)__ldg(L.K + k) * mj;
                        if (L.use_perp) accp += (Acc)__ldg(L.Kps + k) * mj;
                    }
                }
            }
        }
        const Acc scale = (Acc)L.dip_pref * (Acc)L.moment[i] * (Acc)mi;
        double *Eo = E64 ? E64 : L.E_dip, *Epo = Ep64 ? Ep64 : L.E_dip_perp;
        Eo[i] = (double)(scale * acc);
        if (L.use_perp && Epo) Epo[i] = (double)(scale * accp);
    }
}

}  // namespace

namespace {
// resident CTAs of the persistent update kernel with `smem` bytes of dynamic shared memory
template <int VEC>
int persist_grid(int tiles, int64_t smem) {
    int dev = 0, sms = 148, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, dip_update_persist_kernel<VEC>, 32 * UPD_WARPS, (size_t)smem);
    return std::max(1, std::min(tiles, sms * std::max(per, 1)));
}

template <int VEC>
int launch_persist(const HsLattice &L, const HsSwitchList &sw, const int32_t *n_sw_dev, int n_host, int semantics,
                   const HsCounters *C, int tiles, int cap, cudaStream_t st) {
    const int64_t smem = PersistSmem::bytes(cap);
    static int64_t granted = 0;   // dynamic shared memory opted in so far for this variant
    if (smem > 48 * 1024 && smem > granted) {
        cudaError_t e = cudaFuncSetAttribute(dip_update_persist_kernel<VEC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) { hs_set_error("dip_update_persist_kernel: %s", cudaGetErrorString(e)); return HS_ECUDA; }
        granted = smem;
    }
    dip_update_persist_kernel<VEC><<<persist_grid<VEC>(tiles, smem), 32 * UPD_WARPS, (size_t)smem, st>>>(
        L, sw, n_sw_dev, n_host, semantics, C, tiles, cap);
    return hs_check_launch("dip_update_persist_kernel");
}
}  // namespace

int hs_launch_dipolar_update(const HsLattice &L, const HsSwitchList &sw, const int32_t *n_sw_dev, int n_host,
                             int semantics, const HsCounters *C, cudaStream_t st) {
    const bool vec = (L.nx % 4) == 0;
    const int TX = vec ? 128 : 32;
    const int tiles = ((L.nx + TX - 1) / TX) * ((L.ny + UPD_TY - 1) / UPD_TY);
    // a list that fits the shared-memory staging goes to the persistent kernel (a device-side
    // count is bounded by the list's capacity) when the lattice has tiles for at least two
    // waves; smaller lattices give each CTA one tile, where the per-tile kernel's list scan
    // costs less than staging the whole list in every CTA (512^2 pinwheel, Metropolis grid
    // r = 20a: 14.6 -> 13.1 us per step)
    const int most = n_sw_dev ? sw.cap : n_host;
    if (most <= UPD_PLOC && tiles <= 1 << 20 && tiles >= HS_UPD_PERSIST_MIN_TILES) {
        const int cap = std::max(most, 1);
        return vec ? launch_persist<4>(L, sw, n_sw_dev, n_host, semantics, C, tiles, cap, st)
                   : launch_persist<1>(L, sw, n_sw_dev, n_host, semantics, C, tiles, cap, st);
    }
    if (vec) dip_update_kernel<4><<<tiles, 32 * UPD_WARPS, 0, st>>>(L, sw, n_sw_dev, n_host, semantics, C);
    else dip_update_kernel<1><<<tiles, 32 * UPD_WARPS, 0, st>>>(L, sw, n_sw_dev, n_host, semantics, C);
    return hs_check_launch("dip_update_kernel");
}

int hs_launch_dipolar_full_direct(const HsLattice &L, int fp64, double *E64, double *Ep64, cudaStream_t st) {
    const int64_t N = (int64_t)L.nx * L.ny;
    const int threads = 128;
    const int blocks = (int)std::min<int64_t>((N + threads - 1) / threads, 148 * 16);
    const bool full = !L.dip_wrap && L.dip_wy == L.ny - 1 && L.dip_wx == L.nx - 1;
    if (fp64) {
        if (full) dip_full_direct_kernel<double, true><<<blocks, threads, 0, st>>>(L, 1, E64, Ep64);
        else dip_full_direct_kernel<double, false><<<blocks, threads, 0, st>>>(L, 1, E64, Ep64);
    } else {
        if (full) dip_full_direct_kernel<float, true><<<blocks, threads, 0, st>>>(L, 0, E64, Ep64);
        else dip_full_direct_kernel<float, false><<<blocks, threads, 0, st>>>(L, 0, E64, Ep64);
    }
    return hs_check_launch("dip_full_direct_kernel");
}
