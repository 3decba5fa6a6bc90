// (a) incremental dipolar energy update and (b, checker) direct full recompute.
//
// The incremental update is a deterministic gather: the lattice is cut into tiles of
// HS_TY rows x (32*VEC) columns, every CTA keeps the switches whose window reaches its
// tile (in their original order, so the summation order never depends on scheduling),
// and each thread owns VEC consecutive cells of one row: it reads E and mm once (float4
// when the row is 16-byte aligned), accumulates sum_s mm_s * K_s(j - s) over the switches,
// and writes E back once. Semantics follow hotspice/energies.py:310-366:
//   HS_UPDATE_SINGLE   E_j += 2 pref mm_j acc_j; then E_s = -E_s          (update_single)
//   HS_UPDATE_MULTIPLE E_s = -E_s for every switch; E_j += 2 pref mm_j acc_j (update_multiple)
// A switch in "truncated" mode (more than SIMULTANEOUS_SWITCHES_CONVOLUTION_OR_SUM_CUTOFF
// switches on its sublattice, hotspice/energies.py:343-353) contributes only the
// (2k+1)^2 crop of its kernel with wrap (PBC) or zero fill, like convolve2d(..., 'same').
#include "hs_common.cuh"
#include "hs_internal.h"

#include "hs_steps.cuh"

namespace {

template <int VEC>
__global__ void __launch_bounds__(32 * HS_TY)
dip_update_kernel(HsLattice L, HsSwitchList sw, const int32_t *n_sw_dev, int n_host, int semantics,
                  const HsCounters *C) {
    if (C && C->done) return;
    const int nsw = n_sw_dev ? *n_sw_dev : n_host;
    if (nsw <= 0) return;
    constexpr int TX = 32 * VEC;
    const int tiles_x = (L.nx + TX - 1) / TX;
    const int ty0 = (blockIdx.x / tiles_x) * HS_TY;
    const int tx0 = (blockIdx.x % tiles_x) * TX;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int y = ty0 + warp;
    const int x0 = tx0 + lane * VEC;

    __shared__ SwInfo s_sw[HS_LOC];
    __shared__ int s_n;
    float acc[VEC], accp[VEC];
    bool touched[VEC], negate[VEC];
#pragma unroll
    for (int v = 0; v < VEC; ++v) { acc[v] = 0.f; accp[v] = 0.f; touched[v] = false; negate[v] = false; }

    const float pref2 = (float)(2.0 * L.dip_pref);
    __shared__ int s_next;
    for (int base = 0; base < nsw; base = s_next) {
        // Stage, in order, the switches of [base, ...) whose window reaches this tile.
        if (warp == 0) {
            int n = 0, s = base;
            while (s < nsw && n <= HS_LOC - 32) {
                const int k = s + lane;
                bool hit = false;
                SwInfo w{};
                if (k < nsw) {
                    w.y = sw.y[k]; w.x = sw.x[k]; w.mode = sw.mode ? sw.mode[k] : 0;
                    w.sub = hs_sub(L, w.y, w.x);
                    if (w.sub >= 0) {
                        int hy, wy_, hx, wx_;
                        hs_window(L, w.mode, true, hy, wy_);
                        hs_window(L, w.mode, false, hx, wx_);
                        hit = hs_axis_overlap(w.y, hy, wy_, L.ny, ty0, HS_TY) &&
                              hs_axis_overlap(w.x, hx, wx_, L.nx, tx0, TX);
                        w.mm = L.mm[(int64_t)w.y * L.nx + w.x];
                    } else {
                        // no kernel for this unit-cell site: only the sign flip of E applies
                        hit = semantics == HS_UPDATE_MULTIPLE && w.y >= ty0 && w.y < ty0 + HS_TY &&
                              w.x >= tx0 && w.x < tx0 + TX;
                        w.mm = 0.f;
                    }
                }
                const unsigned bal = __ballot_sync(0xffffffffu, hit);
                if (hit) s_sw[n + __popc(bal & ((1u << lane) - 1u))] = w;
                n += __popc(bal);
                s += 32;
            }
            if (lane == 0) { s_n = n; s_next = s; }
        }
        __syncthreads();
        const int n = s_n;
        if (y < L.ny) {
            for (int q = 0; q < n; ++q) {
                const SwInfo w = s_sw[q];
#pragma unroll
                for (int v = 0; v < VEC; ++v) {
                    const int x = x0 + v;
                    if (x >= L.nx) continue;
                    if (w.sub >= 0) {
                        float a = acc[v], ap = accp[v];
                        hs_contrib(L, w, y, x, a, ap);
                        acc[v] = a; accp[v] = ap;
                    }
                    touched[v] = true;
                    if (w.y == y && w.x == x) negate[v] = true;
                }
            }
        }
        __syncthreads();
    }
    if (y >= L.ny) return;
    const int64_t row = (int64_t)y * L.nx;
    if (VEC == 4 && x0 + 3 < L.nx && (L.nx & 3) == 0) {
        bool any = touched[0] || touched[1] || touched[2] || touched[3];
        if (!any) return;
        const float4 mm4 = *reinterpret_cast<const float4 *>(L.mm + row + x0);
        const float mmv[4] = {mm4.x, mm4.y, mm4.z, mm4.w};
        const double2 e01 = *reinterpret_cast<const double2 *>(L.E_dip + row + x0);
        const double2 e23 = *reinterpret_cast<const double2 *>(L.E_dip + row + x0 + 2);
        double ev[4] = {e01.x, e01.y, e23.x, e23.y};
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            if (semantics == HS_UPDATE_MULTIPLE) {
                if (negate[v]) ev[v] = -ev[v];
                ev[v] += (double)(pref2 * (mmv[v] * acc[v]));
            } else {
                ev[v] += (double)(pref2 * (mmv[v] * acc[v]));
                if (negate[v]) ev[v] = -ev[v];
            }
        }
        *reinterpret_cast<double2 *>(L.E_dip + row + x0) = make_double2(ev[0], ev[1]);
        *reinterpret_cast<double2 *>(L.E_dip + row + x0 + 2) = make_double2(ev[2], ev[3]);
        if (L.use_perp) {
            const double2 p01 = *reinterpret_cast<const double2 *>(L.E_dip_perp + row + x0);
            const double2 p23 = *reinterpret_cast<const double2 *>(L.E_dip_perp + row + x0 + 2);
            double pv[4] = {p01.x, p01.y, p23.x, p23.y};
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                if (semantics == HS_UPDATE_MULTIPLE) {
                    if (negate[v]) pv[v] = -pv[v];
                    pv[v] += (double)(pref2 * (mmv[v] * accp[v]));
                } else {
                    pv[v] += (double)(pref2 * (mmv[v] * accp[v]));
                    if (negate[v]) pv[v] = -pv[v];
                }
            }
            *reinterpret_cast<double2 *>(L.E_dip_perp + row + x0) = make_double2(pv[0], pv[1]);
            *reinterpret_cast<double2 *>(L.E_dip_perp + row + x0 + 2) = make_double2(pv[2], pv[3]);
        }
        return;
    }
#pragma unroll
    for (int v = 0; v < VEC; ++v) {
        const int x = x0 + v;
        if (x >= L.nx || !touched[v]) continue;
        const float mmv = L.mm[row + x];
        double e = L.E_dip[row + x];
        if (semantics == HS_UPDATE_MULTIPLE) { if (negate[v]) e = -e; e += (double)(pref2 * (mmv * acc[v])); }
        else { e += (double)(pref2 * (mmv * acc[v])); if (negate[v]) e = -e; }
        L.E_dip[row + x] = e;
        if (L.use_perp) {
            double p = L.E_dip_perp[row + x];
            if (semantics == HS_UPDATE_MULTIPLE) { if (negate[v]) p = -p; p += (double)(pref2 * (mmv * accp[v])); }
            else { p += (double)(pref2 * (mmv * accp[v])); if (negate[v]) p = -p; }
            L.E_dip_perp[row + x] = p;
        }
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

int hs_launch_dipolar_update(const HsLattice &L, const HsSwitchList &sw, const int32_t *n_sw_dev, int n_host,
                             int semantics, const HsCounters *C, cudaStream_t st) {
    const bool vec = (L.nx % 4) == 0;
    const int TX = vec ? 128 : 32;
    const int tiles = ((L.nx + TX - 1) / TX) * ((L.ny + HS_TY - 1) / HS_TY);
    if (vec) dip_update_kernel<4><<<tiles, 32 * HS_TY, 0, st>>>(L, sw, n_sw_dev, n_host, semantics, C);
    else dip_update_kernel<1><<<tiles, 32 * HS_TY, 0, st>>>(L, sw, n_sw_dev, n_host, semantics, C);
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
