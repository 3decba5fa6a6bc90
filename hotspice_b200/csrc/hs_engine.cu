// Persistent cluster engine: many update steps of many lattice instances in one launch.
//
// Each thread-block cluster (CS CTAs, CS in {1, 2, 4, 8, 16}) repeatedly claims an instance
// from a work counter and advances it by its step budget (or until the progress() stop
// rule of hotspice/core.py:753-760 holds), with cluster barriers between the phases of a
// step instead of kernel boundaries:
//   Metropolis: [CTA 0] selection + acceptance + flips (metro_step_cta)  | barrier |
//               [all]   dipolar update of the touched strips              | barrier |
//   Néel:       [all]   barrier/log-time keys of a slice of the cells, CTA argmin -> CTA 0
//                       through distributed shared memory                 | barrier |
//               [CTA 0] final argmin, switching time, flip                | barrier |
//               [all]   dipolar update                                    | barrier |
//   Wolff:      [CTA 0] sparse cluster growth (wolff_step_cta)            | barrier |
// Every branch that decides how many barriers are executed is taken on values every CTA of
// the cluster reads after a barrier, so all CTAs always execute the same barrier sequence.
//
// The dipolar update distributes work items (switch k, window row, 128-column segment) over
// all warps of the cluster. A strip (row, segment) is processed by the item of the first
// switch whose window covers it, which accumulates the contributions of every covering
// switch in list order: each strip is written once, deterministically, and the work is
// proportional to the area the windows touch.
#include <cooperative_groups.h>

#include "hs_steps.cuh"
#include "hs_internal.h"

namespace cg = cooperative_groups;

namespace {

#ifndef HS_ENGINE_THREADS
#define HS_ENGINE_THREADS 512
#endif
#ifndef HS_ENGINE_REGS
#define HS_ENGINE_REGS 128
#endif
#ifndef HS_NEEL_WIN_UNROLL
#define HS_NEEL_WIN_UNROLL 4
#endif
constexpr int ENG_NT = HS_ENGINE_THREADS;   // threads per CTA
constexpr int ENG_MIN_CTAS = 65536 / (ENG_NT * HS_ENGINE_REGS);  // resident CTAs per SM at that register budget
constexpr int ENG_SWCAP = 512;  // switches staged per CTA in shared memory
constexpr int ENG_WS_MAX = HS_ENGINE_WS_MAX;  // largest dynamic shared workspace a launch may ask for

struct SwX {                    // staged switch with its window footprint
    int y, x, mode, sub;
    float mm;
    int ylo, nrows;             // window rows: (ylo + i) mod ny, i < nrows
    int sa0, sa1, sb0, sb1;     // covered 32-column segments: [sa0, sa1) and [sb0, sb1)
};

HS_DEV void footprint(const HsLattice &L, SwX &w) {
    int hy, wy, hx, wx;
    hs_window(L, w.mode, true, hy, wy);
    hs_window(L, w.mode, false, hx, wx);
    const int nseg = (L.nx + 31) >> 5;
    if (wy) {
        if (2 * hy + 1 >= L.ny) { w.ylo = 0; w.nrows = L.ny; }
        else { w.ylo = hs_wrap(w.y - hy, L.ny); w.nrows = 2 * hy + 1; }
    } else {
        const int lo = max(0, w.y - hy), hi = min(L.ny - 1, w.y + hy);
        w.ylo = lo; w.nrows = hi - lo + 1;
    }
    w.sb0 = w.sb1 = 0;
    if (wx && 2 * hx + 1 >= L.nx) { w.sa0 = 0; w.sa1 = nseg; }
    else if (wx) {
        const int lo = w.x - hx, hi = w.x + hx;
        if (lo >= 0 && hi < L.nx) { w.sa0 = lo >> 5; w.sa1 = (hi >> 5) + 1; }
        else if (lo < 0) { w.sa0 = 0; w.sa1 = (hi >> 5) + 1; w.sb0 = (lo + L.nx) >> 5; w.sb1 = nseg; }
        else { w.sa0 = lo >> 5; w.sa1 = nseg; w.sb0 = 0; w.sb1 = ((hi - L.nx) >> 5) + 1; }
        if (w.sb1 > w.sb0 && w.sb0 < w.sa1 && w.sa0 < w.sb1) {  // ranges touch: merge
            w.sa0 = min(w.sa0, w.sb0); w.sa1 = max(w.sa1, w.sb1); w.sb0 = w.sb1 = 0;
        }
    } else {
        const int lo = max(0, w.x - hx), hi = min(L.nx - 1, w.x + hx);
        w.sa0 = lo >> 5; w.sa1 = (hi >> 5) + 1;
    }
}

// Stage the switch list into shared memory with footprints.
HS_DEV int stage_switches(const HsLattice &L, const HsSwitchList &sw, int nsw, SwX *s_sw) {
    const int n = min(nsw, ENG_SWCAP);
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        SwX w;
        w.y = __ldcg(sw.y + k); w.x = __ldcg(sw.x + k); w.mode = sw.mode ? __ldcg(sw.mode + k) : 0;
        w.sub = hs_sub(L, w.y, w.x);
        w.mm = __ldcg(L.mm + (int64_t)w.y * L.nx + w.x);
        footprint(L, w);
        s_sw[k] = w;
    }
    __syncthreads();
    return n;
}

// Contributions of staged switch w to the 4 cells x0..x0+3 of `row`; tch[v] is set for every
// cell inside the switch's window.
HS_DEV void contrib4(const HsLattice &L, const SwX &w, int row, int x0, float acc[4], float accp[4], bool neg[4],
                     bool tch[4]) {
    if (!w.mode && !L.dip_wrap) {
        // exact window without wrapping: one kernel row, consecutive columns
        const int dy = row - w.y;
        if (dy < -L.dip_wy || dy > L.dip_wy) return;
        const int64_t W = 2 * L.dip_wx + 1, H = 2 * L.dip_wy + 1;
        const int64_t base = (int64_t)w.sub * H * W + (int64_t)(dy + L.dip_wy) * W + (L.dip_wx - w.x);
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int x = x0 + v, dx = x - w.x;
            if (x < L.nx && dx >= -L.dip_wx && dx <= L.dip_wx) {
                tch[v] = true;
                acc[v] += w.mm * __ldg(L.K + base + x);
                if (L.use_perp) accp[v] += w.mm * __ldg(L.Kpo + base + x);
            }
            if (dy == 0 && dx == 0) neg[v] = true;
        }
        return;
    }
    SwInfo wi{w.y, w.x, w.mode, w.sub, w.mm};
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const int x = x0 + v;
        if (x >= L.nx) continue;
        tch[v] = true;
        hs_contrib(L, wi, row, x, acc[v], accp[v]);
        if (w.y == row && w.x == x) neg[v] = true;
    }
}

HS_DEV bool covers_seg(const HsLattice &L, const SwX &w, int row, int seg128) {
    int d = row - w.ylo;
    if (d < 0) d += L.ny;
    if (d >= w.nrows) return false;
    // 128-column segment seg128 spans 32-column segments [4 seg128, 4 seg128 + 4)
    const int a0 = 4 * seg128, a1 = a0 + 4;
    return (a0 < w.sa1 && w.sa0 < a1) || (a0 < w.sb1 && w.sb0 < a1);
}

// Dipolar update of the strips covered by the staged switches. Work item = (switch k, one
// row of its window); warps gw = 0..nw-1 of the whole cluster take items gw, gw + nw, ...
// Along the row the warp walks 128-column segments (4 cells per lane). A segment is written
// by the item of the first switch covering it, which accumulates every covering switch in
// list order.
HS_DEV void update_items(const HsLattice &L, const SwX *s_sw, int n, int semantics, int gw, int nw,
                         const HsSwitchList &sw, int nsw_total) {
    if (n == 0) return;
    const int lane = threadIdx.x & 31;
    const float pref2 = (float)(2.0 * L.dip_pref);
    const bool vec = (L.nx & 3) == 0;
    const bool flip_perp = !(L.dip_keep_perp_sign && nsw_total > 1);  // one switch: update_single
    int it0 = 0;
    for (int k = 0; k < n; ++k) {
        const SwX &wk = s_sw[k];
        if (wk.sub < 0) continue;
        const int nr = wk.nrows;
        // first item index of this switch assigned to this warp
        int r = gw - it0;
        r %= nw; if (r < 0) r += nw;
        for (; r < nr; r += nw) {
            int row = wk.ylo + r;
            if (row >= L.ny) row -= L.ny;
            // 128-column segments this switch covers in this row
            const int ranges[2][2] = {{wk.sa0 >> 2, (wk.sa1 + 3) >> 2}, {wk.sb0 >> 2, (wk.sb1 + 3) >> 2}};
            for (int g = 0; g < 2; ++g) {
                for (int seg = ranges[g][0]; seg < ranges[g][1]; ++seg) {
                    if (g == 1 && seg >= ranges[0][0] && seg < ranges[0][1]) continue;  // already done in range 0
                    bool owned = true;
                    for (int q = 0; q < k; ++q)
                        if (s_sw[q].sub >= 0 && covers_seg(L, s_sw[q], row, seg)) { owned = false; break; }
                    if (!owned) continue;  // warp-uniform
                    const int x0 = seg * 128 + lane * 4;
                    float acc[4] = {0.f, 0.f, 0.f, 0.f}, accp[4] = {0.f, 0.f, 0.f, 0.f};
                    bool neg[4] = {false, false, false, false}, tch[4] = {false, false, false, false};
                    for (int q = k; q < n; ++q) {
                        const SwX &w = s_sw[q];
                        if (w.sub < 0 || !covers_seg(L, w, row, seg)) continue;
                        contrib4(L, w, row, x0, acc, accp, neg, tch);
                    }
                    for (int q = n; q < nsw_total; ++q) {  // beyond the staged ones: from global memory
                        SwX w;
                        w.y = __ldcg(sw.y + q); w.x = __ldcg(sw.x + q); w.mode = sw.mode ? __ldcg(sw.mode + q) : 0;
                        w.sub = hs_sub(L, w.y, w.x);
                        if (w.sub < 0) continue;
                        w.mm = __ldcg(L.mm + (int64_t)w.y * L.nx + w.x);
                        footprint(L, w);
                        if (!covers_seg(L, w, row, seg)) continue;
                        contrib4(L, w, row, x0, acc, accp, neg, tch);
                    }
                    // cells that no window reaches keep their energies (E + 0 = E): skip the
                    // read-modify-write of lanes whose 4 cells are all outside the windows
                    if (x0 >= L.nx || !(tch[0] || tch[1] || tch[2] || tch[3])) continue;
                    const int64_t i = (int64_t)row * L.nx + x0;
                    float mv[4];
                    double ev[4], pv[4];
                    if (vec) {
                        const float4 a = __ldcg(reinterpret_cast<const float4 *>(L.mm + i));
                        const double2 e0 = __ldcg(reinterpret_cast<const double2 *>(L.E_dip + i));
                        const double2 e1 = __ldcg(reinterpret_cast<const double2 *>(L.E_dip + i + 2));
                        mv[0] = a.x; mv[1] = a.y; mv[2] = a.z; mv[3] = a.w;
                        ev[0] = e0.x; ev[1] = e0.y; ev[2] = e1.x; ev[3] = e1.y;
                        if (L.use_perp) {
                            const double2 p0 = __ldcg(reinterpret_cast<const double2 *>(L.E_dip_perp + i));
                            const double2 p1 = __ldcg(reinterpret_cast<const double2 *>(L.E_dip_perp + i + 2));
                            pv[0] = p0.x; pv[1] = p0.y; pv[2] = p1.x; pv[3] = p1.y;
                        }
                    } else {
#pragma unroll
                        for (int v = 0; v < 4; ++v) {
                            const bool in = x0 + v < L.nx;
                            mv[v] = in ? __ldcg(L.mm + i + v) : 0.f;
                            ev[v] = in ? __ldcg(L.E_dip + i + v) : 0.0;
                            pv[v] = (in && L.use_perp) ? __ldcg(L.E_dip_perp + i + v) : 0.0;
                        }
                    }
#pragma unroll
                    for (int v = 0; v < 4; ++v) {
                        if (semantics == HS_UPDATE_MULTIPLE) {
                            if (neg[v]) { ev[v] = -ev[v]; if (flip_perp) pv[v] = -pv[v]; }
                            ev[v] += (double)(pref2 * (mv[v] * acc[v]));
                            pv[v] += (double)(pref2 * (mv[v] * accp[v]));
                        } else {
                            ev[v] += (double)(pref2 * (mv[v] * acc[v]));
                            pv[v] += (double)(pref2 * (mv[v] * accp[v]));
                            if (neg[v]) { ev[v] = -ev[v]; pv[v] = -pv[v]; }
                        }
                    }
                    if (vec) {
                        *reinterpret_cast<double2 *>(L.E_dip + i) = make_double2(ev[0], ev[1]);
                        *reinterpret_cast<double2 *>(L.E_dip + i + 2) = make_double2(ev[2], ev[3]);
                        if (L.use_perp) {
                            *reinterpret_cast<double2 *>(L.E_dip_perp + i) = make_double2(pv[0], pv[1]);
                            *reinterpret_cast<double2 *>(L.E_dip_perp + i + 2) = make_double2(pv[2], pv[3]);
                        }
                    } else {
                        for (int v = 0; v < 4 && x0 + v < L.nx; ++v) {
                            L.E_dip[i + v] = ev[v];
                            if (L.use_perp) L.E_dip_perp[i + v] = pv[v];
                        }
                    }
                }
            }
        }
        it0 += nr;
    }
}

// Window update of a single switch (the Néel step): every thread of the cluster takes window
// cells directly (row-major over the window, consecutive threads on consecutive columns) and
// issues the loads of its cells together; the barrier cache is refreshed in the same pass. Per
// cell the arithmetic is that of update_items for one switch (acc = mm_s K, E += 2 pref mm_j acc
// in the same float order, then E_s negated), so the energies are the same bit for bit; cells
// outside the window receive nothing there either.
HS_DEV void update_one(const HsLattice &L, int sy, int sx, float smm, int8_t sm, int t0, int nt, float *cache) {
    const int sub = hs_sub(L, sy, sx);
    if (sub < 0) return;
    int hy, wy, hx, wx;
    hs_window(L, 0, true, hy, wy);
    hs_window(L, 0, false, hx, wx);
    int ylo, nrows, xlo, ncols;
    if (wy) {
        if (2 * hy + 1 >= L.ny) { ylo = 0; nrows = L.ny; } else { ylo = hs_wrap(sy - hy, L.ny); nrows = 2 * hy + 1; }
    } else { ylo = max(0, sy - hy); nrows = min(L.ny - 1, sy + hy) - ylo + 1; }
    if (wx) {
        if (2 * hx + 1 >= L.nx) { xlo = 0; ncols = L.nx; } else { xlo = hs_wrap(sx - hx, L.nx); ncols = 2 * hx + 1; }
    } else { xlo = max(0, sx - hx); ncols = min(L.nx - 1, sx + hx) - xlo + 1; }
    const int total = nrows * ncols;
    const float pref2 = (float)(2.0 * L.dip_pref);
    const bool two = L.use_perp != 0;
    constexpr int U = HS_NEEL_WIN_UNROLL;   // window cells per thread per pass
    // window cell c = r ncols + q of this thread, advanced by nt cells per slot without divisions
    const int dr = nt / ncols, dq = nt - dr * ncols;
    int r0 = t0 / ncols, q0 = t0 - r0 * ncols;
    for (int base = t0; base < total; base += nt * U) {
        int idx[U], rw[U], cl[U];
        float kv[U], kp[U], mv[U], zf[U], zp[U], eb[U];
        double ev[U], pv[U];
        int8_t oc[U], ms[U];
        bool live[U];   // in the window and on a unit-cell site that holds magnets
#pragma unroll
        for (int k = 0; k < U; ++k) {
            const int c = base + k * nt;
            const int r = r0, q = q0;
            r0 += dr; q0 += dq;
            if (q0 >= ncols) { q0 -= ncols; ++r0; }
            int row = ylo + r, col = xlo + q;
            if (row >= L.ny) row -= L.ny;
            if (col >= L.nx) col -= L.nx;
            rw[k] = row; cl[k] = col;
            idx[k] = row * L.nx + col;
            // a site without a kernel never holds a magnet: its energy stays 0 (the reference adds
            // m * ... = 0 there) and the Néel scan never reads its cache entry
            live[k] = c < total && hs_sub(L, row, col) >= 0;
        }
#pragma unroll
        for (int k = 0; k < U; ++k) {
            const bool v = live[k];
            const int i = idx[k];
            kv[k] = v ? hs_kval(L, L.K, sub, rw[k] - sy, cl[k] - sx) : 0.f;
            kp[k] = (v && two) ? hs_kval(L, L.Kpo, sub, rw[k] - sy, cl[k] - sx) : 0.f;
            // the switched cell's new moment and spin come from the handover (smm, sm): its
            // global writes may still be in flight
            const bool src = rw[k] == sy && cl[k] == sx;
            mv[k] = v ? (src ? smm : __ldcg(L.mm + i)) : 0.f;
            ev[k] = v ? __ldcg(L.E_dip + i) : 0.0;
            pv[k] = (v && two) ? __ldcg(L.E_dip_perp + i) : 0.0;
            if (cache) {
                oc[k] = v ? L.occ[i] : (int8_t)0;
                ms[k] = v ? (src ? sm : __ldcg(L.m + i)) : (int8_t)0;
                zf[k] = (v && L.zee) ? __ldg(L.zee + i) : 0.f;
                zp[k] = (v && L.zee && two) ? __ldg(L.zee_perp + i) : 0.f;
                eb[k] = v ? __ldg(L.E_B + i) : 0.f;
            }
        }
#pragma unroll
        for (int k = 0; k < U; ++k) {
            if (!live[k]) continue;
            const int i = idx[k];
            float acc = 0.f, accp = 0.f;
            acc += smm * kv[k];
            if (two) accp += smm * kp[k];
            double e = ev[k] + (double)(pref2 * (mv[k] * acc));
            double p = pv[k] + (double)(pref2 * (mv[k] * accp));
            if (rw[k] == sy && cl[k] == sx) { e = -e; p = -p; }
            L.E_dip[i] = e;
            if (two) L.E_dip_perp[i] = p;
            if (cache) {
                float c = INFINITY;
                if (oc[k]) {
                    const double m = (double)ms[k];
                    double E = e, Ep = p;
                    if (L.zee) { E += m * (double)zf[k]; if (two) Ep += m * (double)zp[k]; }
                    c = neel_cache_value(L, E, two ? Ep : 0.0, (double)eb[k]);
                }
                cache[i] = c;
            }
        }
    }
}

template <int CS>
struct Sync {
    HS_DEV static void all() {
        if constexpr (CS == 1) __syncthreads();
        else cg::this_cluster().sync();
    }
    // all(), with f() run by the threads for which `run` holds between their arrival and their
    // wait (cluster barrier: its release covers only what came before the arrival)
    template <typename F>
    HS_DEV static void all_then(bool run, F f) {
        if constexpr (CS == 1) {
            if (run) f();
            __syncthreads();
        } else {
            asm volatile("barrier.cluster.arrive;" ::: "memory");
            if (run) f();
            asm volatile("barrier.cluster.wait;" ::: "memory");
        }
    }
    HS_DEV static int rank() {
        if constexpr (CS == 1) return 0;
        else return (int)cg::this_cluster().block_rank();
    }
    template <typename T>
    HS_DEV static void publish(T *local, T v) {  // rank 0 thread writes v into every CTA's copy
        if constexpr (CS == 1) *local = v;
        else {
            cg::cluster_group c = cg::this_cluster();
            for (int r = 0; r < CS; ++r) *c.map_shared_rank(local, r) = v;
        }
    }
};

// Block minimum of (key, index); `warp_uniform`: v is already the warp's minimum on every lane.
HS_DEV HsKeyIdx eng_block_kmin(HsKeyIdx v, HsKeyIdx *sm, bool warp_uniform = false) {
    if (!warp_uniform) v = hs_warp_kmin(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sm[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = (lane < (int)(blockDim.x >> 5)) ? sm[lane] : HsKeyIdx{0.0, -1};
        v = hs_warp_kmin(v);
    }
    __syncthreads();
    return v;
}

HS_DEV double eng_block_dmin(double v, double *sm) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sm[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = (lane < (int)(blockDim.x >> 5)) ? sm[lane] : INFINITY;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    }
    __syncthreads();
    return v;
}

HS_DEV MetroScratch metro_scratch_of(const HsLattice &L, const HsGridPlan &P, void *base) {
    int cap, gsz;
    hs_metro_sizes(L, P, cap, gsz);
    char *p = reinterpret_cast<char *>(base);
    MetroScratch S;
    S.cap = cap; S.gsz = gsz;
    S.py = reinterpret_cast<int32_t *>(p); S.px = S.py + cap; p += hs_align_up_d(8LL * cap, 256);
    S.grid = reinterpret_cast<int32_t *>(p); p += hs_align_up_d(4LL * gsz, 256);
    S.ptx = reinterpret_cast<double *>(p); p += hs_align_up_d(8LL * gsz, 256);
    S.pty = reinterpret_cast<double *>(p); p += hs_align_up_d(8LL * gsz, 256);
    S.queue = reinterpret_cast<int32_t *>(p);
    return S;
}

HS_DEV WolffScratch wolff_scratch_of(const HsLattice &L, void *base) {
    const int64_t N = (int64_t)L.nx * L.ny;
    char *p = reinterpret_cast<char *>(base);
    WolffScratch S;
    S.chk_ep = reinterpret_cast<int32_t *>(p); p += hs_align_up_d(4 * N, 256);
    S.cl_ep = reinterpret_cast<int32_t *>(p); p += hs_align_up_d(4 * N, 256);
    S.cl_layer = reinterpret_cast<int32_t *>(p); p += hs_align_up_d(4 * N, 256);
    S.list = reinterpret_cast<int32_t *>(p); p += hs_align_up_d(4 * N, 256);
    S.cand = reinterpret_cast<int32_t *>(p); p += hs_align_up_d(4 * N, 256);
    S.epoch = reinterpret_cast<int32_t *>(p);
    return S;
}

// Shared state of one CTA while it runs an instance.
struct __align__(16) EngShared {
    HsInstance I;                       // the instance descriptor, staged (read through references)
    HsCounters C;                       // rank 0: the instance's counters for the whole run
    unsigned long long call[2];         // Philox call of step st in call[st & 1]
    HsKeyIdx part[16];
    HsKeyIdx red[32];
    double dred[32];
    int inst, n1, y1, x1, m1, nsw;
    int go[2];                          // step st runs while go[st & 1] (double-buffered)
    float mm1;
    int nq[ENG_NT / 32][NEEL_QCAP];     // per-warp candidate queues of the cached Néel scan
    SwX sw[ENG_SWCAP];
};
static_assert(sizeof(HsInstance) % 8 == 0, "HsInstance is copied in 8-byte words");
static_assert(sizeof(HsCounters) % 8 == 0, "HsCounters is copied in 8-byte words");

// Barriers and publication over the CTAs that run the current instance: the whole cluster, or
// this CTA alone (CTA mode). One copy of the step code serves both (a uniform branch per
// barrier), which keeps the kernel's register allocation that of the cluster path.
template <int CS>
struct RunSync {
    bool alone;
    HS_DEV void all() const {
        if (CS == 1 || alone) __syncthreads();
        else Sync<CS>::all();
    }
    template <typename F>
    HS_DEV void all_then(bool run, F f) const {
        if (CS == 1 || alone) { if (run) f(); __syncthreads(); }
        else Sync<CS>::all_then(run, f);
    }
    template <typename T>
    HS_DEV void publish(T *local, T v) const {
        if (CS == 1 || alone) *local = v;
        else Sync<CS>::publish(local, v);
    }
    // rank 0's slot r of a per-CTA array receives v (r = this CTA's rank)
    template <typename T>
    HS_DEV void to_rank0(T *arr, int r, T v) const {
        if constexpr (CS == 1) arr[0] = v;
        else if (alone) arr[0] = v;
        else *cg::this_cluster().map_shared_rank(&arr[r], 0) = v;
    }
};

// Run instance ii to the end of its step budget (or its stop rule) on the whole cluster
// (`rank` = this CTA's rank) or, in CTA mode, on this CTA alone (rank 0).
template <int CS>
HS_DEV void run_instance(EngShared &sh, const HsInstance *insts, int ii, int rank, bool alone, unsigned char *s_ws,
                         int ws_bytes, long long *elapsed_ns) {
    const RunSync<CS> S{alone};
    const int SCS = (CS == 1 || alone) ? 1 : CS;   // CTAs running the instance
    const int warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    const unsigned long long t_claim = hs_globaltimer_ns();   // used by rank 0, thread 0
    {   // stage the instance descriptor in shared memory
        const unsigned long long *src = reinterpret_cast<const unsigned long long *>(insts + ii);
        unsigned long long *dst = reinterpret_cast<unsigned long long *>(&sh.I);
        for (int k = threadIdx.x; k < (int)(sizeof(HsInstance) / 8); k += blockDim.x) dst[k] = __ldg(src + k);
        __syncthreads();
    }
    const HsInstance &I = sh.I;
    const HsLattice &L = sh.I.L;
    const HsSwitchList &sw = sh.I.sw;
    const HsGridPlan &P = sh.I.P;
    // The counters live in rank 0's shared memory while the instance runs (every step reads
    // and updates them) and go back to global memory when it stops; other CTAs receive the
    // values they need (Philox call, switch count) through distributed shared memory.
    HsCounters *const Cg = sh.I.C;
    HsCounters *const C = &sh.C;
    if (rank == 0) {
        const unsigned long long *src = reinterpret_cast<const unsigned long long *>(Cg);
        unsigned long long *dst = reinterpret_cast<unsigned long long *>(&sh.C);
        for (int k = threadIdx.x; k < (int)(sizeof(HsCounters) / 8); k += blockDim.x) dst[k] = __ldcg(src + k);
    }
    __syncthreads();
    const int scheme = sh.I.scheme;
    // progress() runs: at most `budget` steps in this launch; an unfinished run keeps done = 0
    // and the next launch continues it, so every launch ends
    const int64_t budget = I.steps > 0 ? I.steps : (int64_t)HS_PROGRESS_STEPS_MAX;
    // Whether step st runs, and its Philox call, are decided by rank 0's thread 0 as soon as
    // the counters of step st - 1 are final (right after its decision phase) and published
    // to every CTA in slot st & 1; the barriers that end step st - 1 make them visible, so a
    // step needs no barrier of its own for this. Slot st & 1 was last read at the start of
    // step st - 2, before that step's barriers, so the write cannot overtake a read.
    auto decide_next = [&](int64_t next) {
        int go;
        if (C->done) go = 0;
        else if (C->progress) {
            if (C->status || next >= budget) go = 0;   // a failed step, or the budget: not done
            else { go = hs_progress_continue(C, L.n_occ); if (!go) { C->done = 1; C->n_sw = 0; } }
        }
        else go = next < I.steps;
        S.publish(&sh.go[next & 1], go);
        S.publish(&sh.call[next & 1], (unsigned long long)C->rng_call);
    };
    if (rank == 0 && threadIdx.x == 0) decide_next(0);
    S.all();
    for (int64_t st = 0;; ++st) {
        if (!sh.go[st & 1]) break;
        if (scheme == HS_SCHEME_METROPOLIS) {
            if (rank == 0) {
                metro_step_cta(L, C, sw, P, metro_scratch_of(L, P, I.scratch), ws_bytes > 0 ? s_ws : nullptr,
                               ws_bytes);
                __syncthreads();
                if (threadIdx.x == 0) { S.publish(&sh.nsw, C->n_sw); decide_next(st + 1); }
            }
            S.all();
            if (L.has_dipolar) {
                const int nsw = sh.nsw;
                const int n = stage_switches(L, sw, nsw, sh.sw);
                update_items(L, sh.sw, n, HS_UPDATE_MULTIPLE, rank * nwarps + warp, SCS * nwarps, sw, nsw);
            }
            S.all();
        } else if (scheme == HS_SCHEME_NEEL) {
            const uint64_t call = sh.call[st & 1];
            const int64_t N = (int64_t)L.nx * L.ny;
            const int64_t gt = (int64_t)rank * blockDim.x + threadIdx.x, gs = (int64_t)SCS * blockDim.x;
            const bool unif = L.beta_uniform > 0.0;
            double bmin = 0.0;
            if (!unif) {  // b_min pass (hotspice/core.py:688, 696)
                double v = INFINITY;
                for (int64_t i = gt; i < N; i += gs) {
                    if (!L.occ[i]) continue;
                    double b1, b2;
                    hs_barriers(L, (int)(i / L.nx), (int)(i % L.nx), b1, b2);
                    v = fmin(v, fmin(b1, b2));
                }
                v = eng_block_dmin(v, sh.dred);
                if (threadIdx.x == 0) S.to_rank0(sh.part, rank, HsKeyIdx{v, rank});
                S.all();
                if (rank == 0 && threadIdx.x == 0) {
                    double b = INFINITY;
                    for (int r = 0; r < SCS; ++r) b = fmin(b, sh.part[r].key);
                    C->bmin = b;
                    S.publish(&sh.dred[0], b);
                }
                S.all();
                bmin = sh.dred[0];
                S.all();
            }
            const bool two = L.use_perp != 0;
            // barrier cache: uniform beta, no exchange (its neighbours change outside the window)
            float *cache = (unif && !L.has_exchange && I.scratch_bytes >= HS_NEEL_CACHE_OFFSET + 4 * N)
                               ? reinterpret_cast<float *>(reinterpret_cast<char *>(I.scratch) + HS_NEEL_CACHE_OFFSET)
                               : nullptr;
            HsKeyIdx best{0.0, -1};
            if (cache && st > 0) {
                // as many whole warps as give every thread a full chunk of cells (all threads
                // for large lattices): a small lattice is scanned by fewer warps, each with
                // the same chain of loads and exact evaluations as a full one
                const int64_t M = 4 * (int64_t)L.n_occ < 3 * N ? (int64_t)L.n_occ : N;
                const int64_t Pw = min(gs, (M + NEEL_UNR * 32 - 1) / (NEEL_UNR * 32) * 32);
                if (gt - (threadIdx.x & 31) < Pw) best = neel_scan_cached(L, cache, gt, Pw, N, call, best, sh.nq[warp]);
            } else {
                best = neel_scan_range(L, gt, gs, N, call, bmin, best, cache);
            }
            best = eng_block_kmin(best, sh.red, cache && st > 0);
            if (threadIdx.x == 0) S.to_rank0(sh.part, rank, best);
            S.all();
            NeelFlip flip{};   // thread 0 of rank 0: the step's flip, written after the handover
            if (rank == 0 && threadIdx.x == 0) {
                HsKeyIdx w{0.0, -1};
                for (int r = 0; r < SCS; ++r) w = hs_kmin(w, sh.part[r]);
                neel_finalize(L, C, sw, w, call, bmin, unif, two, I.attempt_freq, &flip);
                const int n1 = C->n_sw;
                if (cache && !L.has_dipolar && n1 > 0) {  // no window update: refresh the flipped cell
                    const int64_t i = w.idx;
                    const double m = (double)flip.m_new;
                    double E = 0.0, Ep = 0.0;
                    if (L.zee) { E = m * (double)L.zee[i]; if (two) Ep = m * (double)L.zee_perp[i]; }
                    cache[i] = neel_cache_value(L, E, Ep, (double)L.E_B[i]);
                }
                // hand the switch to every CTA through shared memory (no global round trip)
                S.publish(&sh.n1, n1);
                if (n1 > 0) {
                    S.publish(&sh.y1, flip.y);
                    S.publish(&sh.x1, flip.x);
                    S.publish(&sh.mm1, flip.mm_new);
                    S.publish(&sh.m1, (int)flip.m_new);
                }
                decide_next(st + 1);
            }
            // The flip's global writes (spin, moment, switch list) are issued after this
            // thread's arrival at the barrier, so the barrier does not wait for them: the
            // window update takes the switched cell's new spin and moment from the handover,
            // and the writes are ordered before the next step by the barrier that ends this one.
            S.all_then(rank == 0 && threadIdx.x == 0 && flip.flip, [&] { neel_apply(L, sw, flip); });
            if (L.has_dipolar && sh.n1 > 0)
                update_one(L, sh.y1, sh.x1, sh.mm1, (int8_t)sh.m1, rank * blockDim.x + threadIdx.x, SCS * blockDim.x, cache);
            S.all();
        } else {  // Wolff
            if (rank == 0) {
                wolff_step_cta(L, C, sw, wolff_scratch_of(L, I.scratch));
                __syncthreads();
                if (threadIdx.x == 0) decide_next(st + 1);
            }
            S.all();
        }
    }
    S.all();
    if (rank == 0) {  // counters back to global memory
        const unsigned long long *src = reinterpret_cast<const unsigned long long *>(&sh.C);
        unsigned long long *dst = reinterpret_cast<unsigned long long *>(Cg);
        for (int k = threadIdx.x; k < (int)(sizeof(HsCounters) / 8); k += blockDim.x) dst[k] = src[k];
        // the device time spent on this instance in this launch
        if (elapsed_ns && threadIdx.x == 0) elapsed_ns[ii] = (long long)(hs_globaltimer_ns() - t_claim);
    }
    __syncthreads();
}

// Clusters claim instances from the work counter (rank 0 claims for the cluster). An instance
// flagged HS_INST_ONE_CTA switches the cluster to CTA mode for the rest of the launch: rank 0
// runs that instance alone, every other CTA claims one of its own, and from then on each CTA
// claims and runs instances by itself, with block barriers only. The switch is decided on the
// same flag by every CTA of the cluster, right after the barrier that follows the claim, and
// no cluster barrier or distributed shared memory access follows it, so a CTA may leave the
// launch while the others of its cluster still run. The host lists the flagged instances
// after all others (a flagged instance is never followed by one that needs the cluster; one
// that is still runs correctly, on one CTA).
template <int CS>
__global__ void __launch_bounds__(ENG_NT, ENG_MIN_CTAS) engine_kernel(const HsInstance *insts, int n_inst, int *work,
                                                                      int ws_bytes, long long *elapsed_ns) {
    // dynamic shared workspace (the Poisson-disc sampler's arrays), given only to launches that
    // hold Poisson-disc instances: it takes L1 capacity from the other phases
    extern __shared__ __align__(16) unsigned char s_ws[];
    __shared__ EngShared sh;
    const int rank = Sync<CS>::rank();
    bool alone = false;
    for (;;) {
        int ii;
        if (!alone) {
            if (rank == 0 && threadIdx.x == 0) Sync<CS>::publish(&sh.inst, atomicAdd(work, 1));
            Sync<CS>::all();
            ii = sh.inst;
            if (ii >= n_inst) break;
            if constexpr (CS > 1) {
                if (__ldg(&insts[ii].flags) & HS_INST_ONE_CTA) {
                    alone = true;
                    if (rank != 0) {
                        __syncthreads();   // every thread has read the cluster's claim
                        if (threadIdx.x == 0) sh.inst = atomicAdd(work, 1);
                        __syncthreads();
                        ii = sh.inst;
                        if (ii >= n_inst) break;
                    }
                }
            }
        } else {
            if (threadIdx.x == 0) sh.inst = atomicAdd(work, 1);
            __syncthreads();
            ii = sh.inst;
            if (ii >= n_inst) break;
        }
        run_instance<CS>(sh, insts, ii, alone ? 0 : rank, alone, s_ws, ws_bytes, elapsed_ns);
    }
}

template <int CS>
cudaError_t engine_allow_ws(int bytes) {
    // opt in to the dynamic workspace: static (about 30 KB) plus dynamic shared memory above
    // 48 KB needs it; the largest size granted so far covers every smaller one
    static int granted = 0;
    if (bytes <= granted) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(engine_kernel<CS>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) granted = bytes;
    return e;
}

template <int CS>
int launch_engine(const HsInstance *insts, int n_inst, int *work, int n_clusters, int ws_bytes, long long *elapsed_ns,
                  cudaStream_t st) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(n_clusters * CS, 1, 1);
    cfg.blockDim = dim3(ENG_NT, 1, 1);
    cfg.dynamicSmemBytes = (size_t)ws_bytes;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CS;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (CS > 8) {
        cudaError_t e = cudaFuncSetAttribute(engine_kernel<CS>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) { hs_set_error("engine: cluster size %d not allowed: %s", CS, cudaGetErrorString(e)); return HS_ECUDA; }
    }
    {
        cudaError_t e = engine_allow_ws<CS>(ws_bytes);
        if (e != cudaSuccess) { hs_set_error("engine: shared workspace: %s", cudaGetErrorString(e)); return HS_ECUDA; }
    }
    cudaError_t e = cudaLaunchKernelEx(&cfg, engine_kernel<CS>, insts, n_inst, work, ws_bytes, elapsed_ns);
    if (e != cudaSuccess) { hs_set_error("engine launch (cluster %d x %d): %s", CS, n_clusters, cudaGetErrorString(e)); return HS_ECUDA; }
    return hs_check_launch("engine_kernel");
}

}  // namespace

int hs_launch_engine(const HsInstance *insts, int n_inst, int cluster_size, int n_clusters, int *work, int ws_bytes,
                     long long *elapsed_ns, cudaStream_t st) {
    if (ws_bytes < 0 || ws_bytes > ENG_WS_MAX) {
        hs_set_error("engine: shared workspace of %d bytes outside [0, %d]", ws_bytes, ENG_WS_MAX);
        return HS_EINVAL;
    }
    cudaError_t e = cudaMemsetAsync(work, 0, sizeof(int), st);
    if (e != cudaSuccess) { hs_set_error("engine: work counter reset: %s", cudaGetErrorString(e)); return HS_ECUDA; }
    switch (cluster_size) {
        case 1: return launch_engine<1>(insts, n_inst, work, n_clusters, ws_bytes, elapsed_ns, st);
        case 2: return launch_engine<2>(insts, n_inst, work, n_clusters, ws_bytes, elapsed_ns, st);
        case 4: return launch_engine<4>(insts, n_inst, work, n_clusters, ws_bytes, elapsed_ns, st);
        case 8: return launch_engine<8>(insts, n_inst, work, n_clusters, ws_bytes, elapsed_ns, st);
        case 16: return launch_engine<16>(insts, n_inst, work, n_clusters, ws_bytes, elapsed_ns, st);
        default: hs_set_error("engine: cluster size must be 1, 2, 4, 8 or 16"); return HS_EINVAL;
    }
}

int hs_engine_max_clusters_impl(int cluster_size) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cluster_size, 1, 1);
    cfg.blockDim = dim3(ENG_NT, 1, 1);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cluster_size;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    cudaError_t e;
    switch (cluster_size) {
        case 1: e = cudaOccupancyMaxActiveClusters(&n, engine_kernel<1>, &cfg); break;
        case 2: e = cudaOccupancyMaxActiveClusters(&n, engine_kernel<2>, &cfg); break;
        case 4: e = cudaOccupancyMaxActiveClusters(&n, engine_kernel<4>, &cfg); break;
        case 8: e = cudaOccupancyMaxActiveClusters(&n, engine_kernel<8>, &cfg); break;
        case 16:
            cudaFuncSetAttribute(engine_kernel<16>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
            e = cudaOccupancyMaxActiveClusters(&n, engine_kernel<16>, &cfg); break;
        default: hs_set_error("engine: bad cluster size"); return HS_EINVAL;
    }
    if (e != cudaSuccess) { hs_set_error("cudaOccupancyMaxActiveClusters: %s", cudaGetErrorString(e)); return HS_ECUDA; }
    return n;
}
