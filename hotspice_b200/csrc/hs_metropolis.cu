// (d) Metropolis multisample step (hotspice/core.py:659-677) with the selection schemes of
// Magnets.select (core.py:456-570): 'grid' (supercells every second one, random offset, one
// random occupied cell per supercell), 'single', and Poisson-disc dart throwing
// (hotspice/poisson.py:72-128) run in cell units.
//
// One CTA performs selection, the occupation filter (retrying like select() does), the
// acceptance test p = clip(exp(-dE beta), 1e-10, 1e10) > u, the flips, and writes the switch
// list with the per-sublattice branch choice of DipolarEnergy.update_multiple (more than
// SIMULTANEOUS_SWITCHES_CONVOLUTION_OR_SUM_CUTOFF switches -> truncated window). The
// dipolar gather update (hs_dipolar.cu) then consumes the list. Every variate comes from the
// Philox call sequence the reference would consume: offset x, offset y, supercell picks,
// [METROPOLIS_TIME draws], acceptance draws; retries and fallbacks add calls in order.
#include "hs_common.cuh"
#include "hs_internal.h"

namespace {

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

// Poisson-disc dart throwing in cell units, executed by warp 0. Returns the number of points
// written to (py, px) as nearest cell indices, and advances `call` by the variates consumed.
HS_DEV int poisson_warp(const HsLattice &L, const HsGridPlan &P, const MetroScratch &S, uint64_t &call, int *status) {
    const int lane = threadIdx.x & 31;
    const double width = L.nx, height = L.ny;
    const double r = P.r_cells + 1.0;
    const double cs = r / sqrt(2.0);
    const double rSq = r * r;
    const int gw = (int)ceil(width / cs), gh = (int)ceil(height / cs);
    const int gsz = gw * gh;
    if (gsz > S.gsz) { if (lane == 0) *status |= HS_ST_POISSON_OVERFLOW; return 0; }
    for (int g = lane; g < gsz; g += 32) S.grid[g] = -1;
    __syncwarp();
    auto rnd = [&]() { const double u = hs_u53(L.seed, call, 0u); call += 1; return u; };
    const double p0x = (double)(int)(width * rnd());
    const double p0y = (double)(int)(height * rnd());
    int npts = 1, nq = 1;
    if (lane == 0) { S.ptx[0] = p0x; S.pty[0] = p0y; S.queue[0] = 0; S.grid[(int)(p0x / cs) + (int)(p0y / cs) * gw] = 0; }
    __syncwarp();
    while (nq > 0) {
        const int qi = (int)(rnd() * nq);
        const int q = S.queue[qi];
        // list.pop(qi): shift the tail left, preserving order
        for (int j = qi + lane; j < nq - 1; j += 32) {
            const int v = S.queue[j + 1];
            __syncwarp(__activemask());
            S.queue[j] = v;
        }
        __syncwarp();
        nq -= 1;
        const double qx = S.ptx[q], qy = S.pty[q];
        for (int t = 0; t < P.poisson_k; ++t) {
            const double alpha = 6.283185307179586 * rnd();
            const double d = r * sqrt(3.0 * rnd() + 1.0);
            const double px = qx + d * cos(alpha);
            const double py = qy + d * sin(alpha);
            if (!(0.0 <= px && px < width && 0.0 <= py && py < height)) continue;
            const int gx = (int)(px / cs), gy = (int)(py / cs);
            bool conflict = false;
            if (lane < 25) {
                const int xx = gx - 2 + lane / 5, yy = gy - 2 + lane % 5;
                const int g = S.grid[pymod(xx + yy * gw, gsz)];
                if (g >= 0) {
                    double dx = fabs(px - S.ptx[g]), dy = fabs(py - S.pty[g]);
                    if (dx > width * 0.5) dx -= width;
                    if (dy > height * 0.5) dy -= height;
                    conflict = (dx * dx + dy * dy) <= rSq;
                }
            }
            if (__any_sync(0xffffffffu, conflict)) continue;
            if (npts >= S.gsz) { if (lane == 0) *status |= HS_ST_POISSON_OVERFLOW; break; }
            if (lane == 0) {
                S.ptx[npts] = px; S.pty[npts] = py;
                S.queue[nq] = npts;
                S.grid[gx + gy * gw] = npts;
            }
            __syncwarp();
            npts += 1; nq += 1;
        }
    }
    __syncwarp();
    // keep points with x < max(r, w - r), y < max(r, h - r) (PBC=True default), then offset
    const double lx = fmax(r, width - r), ly = fmax(r, height - r);
    const double ox = (double)(int)(rnd() * width), oy = (double)(int)(rnd() * height);
    if (lane == 0) {
        int k = 0;
        for (int g = 0; g < gsz; ++g) {
            const int p = S.grid[g];
            if (p < 0) continue;
            const double x = S.ptx[p], y = S.pty[p];
            if (!(x >= 0.0 && y >= 0.0 && x < lx && y < ly)) continue;
            const double fx = fmod(x + ox, width), fy = fmod(y + oy, height);
            // nearest cell index, ties to the lower index
            int ix = (int)floor(fx); if (fx - ix > 0.5) ix += 1; ix = min(max(ix, 0), L.nx - 1);
            int iy = (int)floor(fy); if (fy - iy > 0.5) iy += 1; iy = min(max(iy, 0), L.ny - 1);
            if (k < S.cap) { S.py[k] = iy; S.px[k] = ix; }
            ++k;
        }
        if (k > S.cap) { *status |= HS_ST_POISSON_OVERFLOW; k = S.cap; }
        S.grid[0] = k;  // hand the count back through memory
    }
    __syncwarp();
    return S.grid[0];
}

__global__ void __launch_bounds__(MT) metropolis_kernel(HsLattice L, HsCounters *C, HsSwitchList sw, HsGridPlan P,
                                                        MetroScratch S) {
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
                const int n = poisson_warp(L, P, S, c, &st);
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
    if (threadIdx.x < 256) s_bins[threadIdx.x] = 0;
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

}  // namespace

static void metro_sizes(const HsLattice &L, const HsGridPlan &P, int &cap, int &gsz) {
    cap = std::max(P.n_sc, 1);
    gsz = 0;
    if (P.sample_scheme == HS_SAMPLE_POISSON) {
        const double r = P.r_cells + 1.0, cs = r / sqrt(2.0);
        gsz = (int)(ceil(L.nx / cs) * ceil(L.ny / cs));
        cap = std::max(cap, gsz);
    }
}

int64_t hs_metropolis_scratch(const HsLattice &L, const HsGridPlan &P) {
    int cap, gsz;
    metro_sizes(L, P, cap, gsz);
    return hs_align_up(8LL * cap, 256) + hs_align_up(4LL * gsz, 256) + 2 * hs_align_up(8LL * gsz, 256) +
           hs_align_up(4LL * gsz + 4, 256) + 256;
}

int hs_launch_metropolis(const HsLattice &L, HsCounters *C, const HsSwitchList &sw, const HsGridPlan &P,
                         void *scratch, int64_t scratch_bytes, cudaStream_t st) {
    int cap, gsz;
    metro_sizes(L, P, cap, gsz);
    if (scratch_bytes < hs_metropolis_scratch(L, P)) {
        hs_set_error("hs_metropolis_step: scratch %lld < %lld bytes", (long long)scratch_bytes,
                     (long long)hs_metropolis_scratch(L, P));
        return HS_ENOMEM;
    }
    if (L.ux * L.uy > 256) { hs_set_error("hs_metropolis_step: unit cell larger than 256 sites"); return HS_ERANGE; }
    if (sw.cap < 1) { hs_set_error("hs_metropolis_step: switch list capacity < 1"); return HS_EINVAL; }
    char *p = reinterpret_cast<char *>(scratch);
    MetroScratch S;
    S.cap = cap;
    S.gsz = gsz;
    S.py = reinterpret_cast<int32_t *>(p);
    S.px = S.py + cap;
    p += hs_align_up(8LL * cap, 256);
    S.grid = reinterpret_cast<int32_t *>(p); p += hs_align_up(4LL * gsz, 256);
    S.ptx = reinterpret_cast<double *>(p); p += hs_align_up(8LL * gsz, 256);
    S.pty = reinterpret_cast<double *>(p); p += hs_align_up(8LL * gsz, 256);
    S.queue = reinterpret_cast<int32_t *>(p);
    if (P.sample_scheme == HS_SAMPLE_POISSON && gsz < 1) { hs_set_error("Poisson grid empty"); return HS_EINVAL; }
    metropolis_kernel<<<1, MT, 0, st>>>(L, C, sw, P, S);
    int rc = hs_check_launch("metropolis_kernel");
    if (rc) return rc;
    if (L.has_dipolar) return hs_launch_dipolar_update(L, sw, &C->n_sw, 0, HS_UPDATE_MULTIPLE, C, st);
    return HS_OK;
}

// ---------------------------------------------------------------------------------------
// Allocation-free variant of hs_metropolis_step.
//
// Some callers cannot hand this library a scratch buffer: they own no device allocator
// (an embedding application that passes in only its state arrays and forbids further device
// allocations under a fixed memory budget, or a real-time host loop that must never call
// cudaMalloc, whose implicit synchronisation it cannot afford). For them the candidate and
// Poisson-disc working arrays live in one fixed file-scope device array instead. The array
// exists once per GPU that loads this library and stays allocated until the process exits.
// The first call on a device, made with that device current, looks up the array's device
// address with cudaGetSymbolAddress; make that first call before any stream capture. Every
// call shares the array and it keeps the previous call's contents: the kernel rewrites
// every entry it reads (nothing has to start at zero), and calls that overlap on the GPU
// (other streams, other threads) race on it.
// ---------------------------------------------------------------------------------------
#include <mutex>

#define HS_NOALLOC_METRO_BYTES (4LL << 20)   // 4 MiB
#define HS_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) unsigned char g_hs_metro_scratch[HS_NOALLOC_METRO_BYTES];
static void *g_hs_metro_scratch_ptr[HS_NOALLOC_MAX_DEVICES];
static std::mutex g_hs_metro_scratch_mu;

extern "C" int hs_metropolis_step_noalloc(const HsLattice *L, HsCounters *C, const HsSwitchList *sw,
                                          const HsGridPlan *P, void *stream) {
    if (!L || !C || !sw || !P) { hs_set_error("hs_metropolis_step_noalloc: null argument"); return HS_EINVAL; }
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) { hs_set_error("hs_metropolis_step_noalloc: cudaGetDevice: %s", cudaGetErrorString(e)); return HS_ECUDA; }
    if (dev < 0 || dev >= HS_NOALLOC_MAX_DEVICES) {
        hs_set_error("hs_metropolis_step_noalloc: device %d beyond the %d supported", dev, HS_NOALLOC_MAX_DEVICES);
        return HS_ERANGE;
    }
    void *ptr;
    {
        std::lock_guard<std::mutex> lock(g_hs_metro_scratch_mu);
        ptr = g_hs_metro_scratch_ptr[dev];
        if (!ptr) {  // set-up: once per device, with that device current
            e = cudaGetSymbolAddress(&ptr, g_hs_metro_scratch);
            if (e != cudaSuccess || !ptr) {
                hs_set_error("hs_metropolis_step_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
                return HS_ECUDA;
            }
            g_hs_metro_scratch_ptr[dev] = ptr;
        }
    }
    if (L->nx <= 0 || L->ny <= 0) { hs_set_error("hs_metropolis_step_noalloc: bad lattice size"); return HS_EINVAL; }
    const int64_t need = hs_metropolis_scratch(*L, *P);
    if (need > HS_NOALLOC_METRO_BYTES) {
        hs_set_error("hs_metropolis_step_noalloc: this selection plan needs %lld bytes of scratch, the fixed "
                     "scratch holds %lld; use hs_metropolis_step with a caller-provided buffer",
                     (long long)need, (long long)HS_NOALLOC_METRO_BYTES);
        return HS_ERANGE;
    }
    return hs_metropolis_step(L, C, sw, P, ptr, HS_NOALLOC_METRO_BYTES, stream);
}
