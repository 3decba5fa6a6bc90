// Relaxation to a (meta)stable state: Magnets._minimize_all / relax / minimize
// (hotspice/core.py:763-861).
//
// _minimize_all (one "sweep"): the lattice is cut into (2 ux) x (2 uy) interleaved subgrids
// (one subgrid when simultaneous), visited in a random order. In each subgrid every magnet
// whose switch lowers the energy (switch_energy < 0; or switch_energy / 2 + E_B < 0 when the
// barrier is not ignored) switches at once, and the energies are updated before the next
// subgrid is decided. On the device a sweep is:
//   relax_perm_kernel      the subgrid order: stable argsort of one Philox call of P variates
//   per subgrid i:
//     relax_decide_kernel  switch decisions (from E before any flip of this subgrid), a flag
//                          per candidate and a count per block
//     relax_apply_kernel   order-preserving compaction into the switch list, the flips, the
//                          counters; the list's truncated-window flag follows
//                          DipolarEnergy.update_multiple's per-sublattice rule
//     dip_update_kernel    (hs_dipolar.cu) consumes the list
// relax() adds, after every sweep, its stop rule: nothing switched, the state equals the one
// two sweeps before, or int(sqrt(nx^2 + ny^2)) sweeps (relax_compare_kernel, relax_end_kernel).
// Every kernel reads the control state from device memory and returns at once when the stop
// rule has fired, so the host can enqueue (or replay as a CUDA graph) several sweeps and look
// at the state once.
//
// minimize() (sequential): per iteration the switch energy of every cell, the number n of
// magnets gaining more than kBT and the first argmin. If n > 0, ceil(0.3 n) of those n switch:
// the ones with the smallest Philox keys of one call over n elements (the stream's
// choice(n, k, replace=False)), found exactly by a 5-pass radix select on the 53-bit keys;
// else the argmin switches if it lowers the energy and was not picked three times.
#include "hs_common.cuh"
#include "hs_internal.h"

namespace {

constexpr int RX_T = 256;               // threads per block of the grid kernels
constexpr int RX_PER = 4;               // candidates per thread
constexpr int RX_CH = RX_T * RX_PER;    // candidates per block
constexpr int RX_MAX_P = 1024;          // subgrids per sweep (4 * 256 unit-cell sites)
constexpr int RX_MAX_U = 256;           // unit-cell sites
constexpr int MN_PASSES = 5;            // radix-select passes over the 53-bit keys
constexpr int MN_BINS = 2048;           // largest digit (11 bits)
__constant__ int c_mn_lo[MN_PASSES] = {42, 31, 20, 10, 0};
__constant__ int c_mn_bits[MN_PASSES] = {11, 11, 11, 10, 10};

struct RelaxState {
    int32_t done;       // stop rule fired: the remaining kernels of the sweep do nothing
    int32_t sweep;      // sweeps completed (relax)
    int32_t differs;    // the state after this sweep differs from the one two sweeps before
    int32_t pad0;
    int64_t sw_start;   // C->switches when the sweep began
    // minimize()
    int32_t mode;       // 0: stop, 1: the argmin switches, 2: ceil(frac n) of n switch
    int32_t count;      // n
    int32_t k;          // ceil(frac n)
    int32_t k_rem;      // radix select: how many keys equal to the threshold are taken
    int32_t eq_total;   // keys equal to the threshold
    int32_t imin;
    uint64_t prefix;    // radix select: threshold key bits found so far
    uint64_t call;      // Philox call of the choice
    double vmin;
};

struct RelaxBufs {
    RelaxState *st;
    int32_t *order;      // RX_MAX_P
    int32_t *blk;        // per-block counts
    int32_t *blk2;       // second per-block array (minimize: equal-key counts)
    double *blk_v;       // minimize: per-block minimum
    int32_t *blk_i;      //           and its index
    int32_t *sub_counts; // RX_MAX_U
    uint8_t *flags;      // N
    int8_t *snap;        // 2 N (relax) / visited N (minimize)
    int32_t *cells;      // N (minimize)
    int32_t *hist;       // MN_PASSES * MN_BINS (minimize)
};

HS_DEV uint64_t u53_bits(uint64_t seed, uint64_t call, uint32_t e) {
    HsU4 w = hs_philox(e, (uint32_t)call, (uint32_t)(call >> 32), 0u, (uint32_t)seed, (uint32_t)(seed >> 32));
    return ((uint64_t)(w.x >> 5) << 26) | (uint64_t)(w.y >> 6);
}

// Exclusive prefix of v over the block (RX_T threads) and the block total.
HS_DEV int block_scan(int v, int &total, int *s_w) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_w[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int w = lane < RX_T / 32 ? s_w[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < RX_T / 32) s_w[lane] = w;   // inclusive warp prefix
    }
    __syncthreads();
    total = s_w[RX_T / 32 - 1];
    const int before = warp ? s_w[warp - 1] : 0;
    __syncthreads();
    return before + x - v;
}

HS_DEV int block_sum(int v, int *s_w) {
    int t;
    block_scan(v, t, s_w);
    return t;
}

HS_DEV double kbt_at(const HsLattice &L, int64_t i) {
    const double b = hs_beta(L, i);
    return 1.0 / b;     // beta = inf (T = 0) gives kBT = 0
}

// ---------------------------------------------------------------------------------------
// _minimize_all / relax
// ---------------------------------------------------------------------------------------
struct Subgrid {
    int y0, x0, nys, nxs, M;
    bool active;
};

HS_DEV Subgrid subgrid(const HsLattice &L, const RelaxBufs &B, int i, int sx, int sy) {
    Subgrid g;
    const int o = B.order[i];
    if (o < 0 || o >= sx * sy) {   // no order drawn for this layout: an empty subgrid
        g.y0 = g.x0 = g.nys = g.nxs = g.M = 0;
        g.active = false;
        return g;
    }
    g.y0 = o / sx;
    g.x0 = o % sx;
    g.active = L.occ[(int64_t)g.y0 * L.nx + g.x0] != 0;
    g.nys = (L.ny - g.y0 + sy - 1) / sy;
    g.nxs = (L.nx - g.x0 + sx - 1) / sx;
    g.M = g.nys * g.nxs;
    return g;
}

__global__ void __launch_bounds__(1024) relax_perm_kernel(HsLattice L, HsCounters *C, RelaxBufs B, int P) {
    __shared__ uint64_t s_key[RX_MAX_P];
    if (B.st->done) return;
    const uint64_t call = C->rng_call;
    for (int e = threadIdx.x; e < P; e += blockDim.x) s_key[e] = u53_bits(L.seed, call, (uint32_t)e);
    __syncthreads();
    for (int e = threadIdx.x; e < P; e += blockDim.x) {
        const uint64_t k = s_key[e];
        int rank = 0;
        for (int j = 0; j < P; ++j) rank += (s_key[j] < k) || (s_key[j] == k && j < e);
        B.order[rank] = e;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        C->rng_call = call + 1;
        B.st->sw_start = C->switches;
    }
}

__global__ void __launch_bounds__(RX_T) relax_decide_kernel(HsLattice L, RelaxBufs B, int i, int sx, int sy,
                                                            int ignore_barrier, int simultaneous) {
    __shared__ int s_w[RX_T / 32];
    if (B.st->done) return;
    const Subgrid g = subgrid(L, B, i, sx, sy);
    int cnt = 0;
#pragma unroll
    for (int k = 0; k < RX_PER; ++k) {
        const int t = blockIdx.x * RX_CH + k * RX_T + threadIdx.x;
        if (t >= g.M) continue;
        uint8_t f = 0;
        if (g.active) {
            const int y = g.y0 + (t / g.nxs) * sy, x = g.x0 + (t % g.nxs) * sx;
            double E, Ep;
            hs_energy_at(L, y, x, E, Ep);
            const double dE = -2.0 * E;
            f = ignore_barrier ? (dE < 0.0) : (dE / 2.0 + (double)L.E_B[(int64_t)y * L.nx + x] < 0.0);
            if (f && simultaneous) atomicAdd(&B.sub_counts[(y % L.uy) * L.ux + (x % L.ux)], 1);
        }
        B.flags[t] = f;
        cnt += f;
    }
    cnt = block_sum(cnt, s_w);
    if (threadIdx.x == 0) B.blk[blockIdx.x] = cnt;
}

__global__ void __launch_bounds__(RX_T) relax_apply_kernel(HsLattice L, HsCounters *C, RelaxBufs B, HsSwitchList sw,
                                                           int i, int sx, int sy, int simultaneous, int nblk) {
    __shared__ int s_w[RX_T / 32];
    if (B.st->done) {
        if (blockIdx.x == 0 && threadIdx.x == 0) C->n_sw = 0;
        return;
    }
    const Subgrid g = subgrid(L, B, i, sx, sy);
    // offset of this block and the subgrid total
    int before = 0, all = 0;
    for (int j = threadIdx.x; j < nblk; j += RX_T) {
        const int c = B.blk[j];
        all += c;
        if (j < (int)blockIdx.x) before += c;
    }
    before = block_sum(before, s_w);
    all = block_sum(all, s_w);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        C->n_sw = all;
        C->switches += all;
        C->attempted += all;
    }
    int pos = before;
#pragma unroll 1
    for (int k = 0; k < RX_PER; ++k) {
        const int t = blockIdx.x * RX_CH + k * RX_T + threadIdx.x;
        const int f = (t < g.M) ? B.flags[t] : 0;
        int tot;
        const int p = pos + block_scan(f, tot, s_w);
        if (f) {
            const int y = g.y0 + (t / g.nxs) * sy, x = g.x0 + (t % g.nxs) * sx;
            const int64_t c = (int64_t)y * L.nx + x;
            const int cnt = simultaneous ? B.sub_counts[(y % L.uy) * L.ux + (x % L.ux)] : all;
            sw.y[p] = y;
            sw.x[p] = x;
            if (sw.mode) sw.mode[p] = cnt > L.trunc_cutoff ? 1 : 0;
            L.m[c] = (int8_t)(-L.m[c]);
            L.mm[c] = -L.mm[c];
        }
        pos += tot;
    }
}

__global__ void __launch_bounds__(RX_T) relax_compare_kernel(HsLattice L, const HsCounters *C, RelaxBufs B) {
    __shared__ int s_w[RX_T / 32];
    if (B.st->done || C->switches == B.st->sw_start) return;
    const int64_t N = (int64_t)L.nx * L.ny;
    int8_t *snap = B.snap + ((B.st->sweep + 1) & 1) * N;
    int d = 0;
    for (int64_t c = (int64_t)blockIdx.x * RX_T + threadIdx.x; c < N; c += (int64_t)gridDim.x * RX_T) {
        const int8_t a = L.m[c];
        d |= a != snap[c];
        snap[c] = a;
    }
    d = block_sum(d, s_w);
    if (threadIdx.x == 0 && d) atomicOr(&B.st->differs, 1);
}

__global__ void relax_end_kernel(const HsCounters *C, RelaxBufs B, int n_max) {
    RelaxState *s = B.st;
    if (s->done) return;
    const int n = ++s->sweep;
    if (C->switches == s->sw_start) s->done = 1;       // nothing changed
    else if (!s->differs) s->done = 1;                 // 2-cycle
    else if (n >= n_max) s->done = 1;
    s->differs = 0;
}

// ---------------------------------------------------------------------------------------
// minimize
// ---------------------------------------------------------------------------------------
__global__ void __launch_bounds__(RX_T) mn_scan_kernel(HsLattice L, RelaxBufs B) {
    __shared__ int s_w[RX_T / 32];
    __shared__ double s_v[RX_T];
    __shared__ int s_i[RX_T];
    if (B.st->done) return;
    const int64_t N = (int64_t)L.nx * L.ny;
    int cnt = 0;
    double vmin = INFINITY;
    int imin = INT32_MAX;
#pragma unroll
    for (int k = 0; k < RX_PER; ++k) {
        const int64_t c = (int64_t)blockIdx.x * RX_CH + k * RX_T + threadIdx.x;
        if (c >= N) continue;
        const int y = (int)(c / L.nx), x = (int)(c % L.nx);
        double E, Ep;
        hs_energy_at(L, y, x, E, Ep);
        const double dE = -2.0 * E;
        const uint8_t f = dE < -kbt_at(L, c);
        B.flags[c] = f;
        cnt += f;
        if (dE < vmin) { vmin = dE; imin = (int)c; }   // increasing c: first occurrence kept
    }
    cnt = block_sum(cnt, s_w);
    s_v[threadIdx.x] = vmin;
    s_i[threadIdx.x] = imin;
    __syncthreads();
    for (int o = RX_T / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            const double v2 = s_v[threadIdx.x + o];
            const int i2 = s_i[threadIdx.x + o];
            if (v2 < s_v[threadIdx.x] || (v2 == s_v[threadIdx.x] && i2 < s_i[threadIdx.x])) {
                s_v[threadIdx.x] = v2;
                s_i[threadIdx.x] = i2;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        B.blk[blockIdx.x] = cnt;
        B.blk_v[blockIdx.x] = s_v[0];
        B.blk_i[blockIdx.x] = s_i[0];
    }
}

__global__ void __launch_bounds__(1024) mn_decide_kernel(HsLattice L, HsCounters *C, RelaxBufs B, HsSwitchList sw,
                                                         int nblk, double frac) {
    __shared__ long long s_cnt[32];
    __shared__ double s_v[1024];
    __shared__ int s_i[1024];
    RelaxState *s = B.st;
    if (s->done) {   // the update that follows must see an empty list
        if (threadIdx.x == 0) C->n_sw = 0;
        return;
    }
    long long cnt = 0;
    double vmin = INFINITY;
    int imin = INT32_MAX;
    for (int j = threadIdx.x; j < nblk; j += blockDim.x) {
        cnt += B.blk[j];
        const double v = B.blk_v[j];
        const int ii = B.blk_i[j];
        if (v < vmin || (v == vmin && ii < imin)) { vmin = v; imin = ii; }
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0) s_cnt[threadIdx.x >> 5] = cnt;
    s_v[threadIdx.x] = vmin;
    s_i[threadIdx.x] = imin;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            const double v2 = s_v[threadIdx.x + o];
            const int i2 = s_i[threadIdx.x + o];
            if (v2 < s_v[threadIdx.x] || (v2 == s_v[threadIdx.x] && i2 < s_i[threadIdx.x])) {
                s_v[threadIdx.x] = v2;
                s_i[threadIdx.x] = i2;
            }
        }
        __syncthreads();
    }
    // zero the radix-select histograms and the sublattice counts for this iteration
    for (int j = threadIdx.x; j < MN_PASSES * MN_BINS; j += blockDim.x) B.hist[j] = 0;
    for (int j = threadIdx.x; j < RX_MAX_U; j += blockDim.x) B.sub_counts[j] = 0;
    if (threadIdx.x != 0) return;
    long long total = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) total += s_cnt[w];
    s->vmin = s_v[0];
    s->imin = s_i[0];
    if (total > 0) {
        s->mode = 2;
        s->count = (int)total;
        s->k = (int)ceil((double)total * frac);
        s->k_rem = s->k;
        s->prefix = 0;
        s->call = C->rng_call;
        C->rng_call += 1;
        return;
    }
    s->mode = 0;
    C->n_sw = 0;
    const int c = s->imin;
    if (!(s->vmin < 0.0) || c == INT32_MAX) { s->done = 1; return; }   // no switch lowers the energy
    const int vis = ++B.snap[c];
    if (vis >= 3) { s->done = 1; return; }
    s->mode = 1;
    const int y = c / L.nx, x = c % L.nx;
    sw.y[0] = y;
    sw.x[0] = x;
    if (sw.mode) sw.mode[0] = 0;
    L.m[c] = (int8_t)(-L.m[c]);
    L.mm[c] = -L.mm[c];
    C->n_sw = 1;
    C->switches += 1;
    C->attempted += 1;
}

// Ordered list of the cells that gain more than kBT (row-major, as numpy.where gives them).
__global__ void __launch_bounds__(RX_T) mn_compact_kernel(HsLattice L, RelaxBufs B, int nblk) {
    __shared__ int s_w[RX_T / 32];
    if (B.st->done || B.st->mode != 2) return;
    const int64_t N = (int64_t)L.nx * L.ny;
    int before = 0;
    for (int j = threadIdx.x; j < (int)blockIdx.x; j += RX_T) before += B.blk[j];
    int pos = block_sum(before, s_w);
#pragma unroll 1
    for (int k = 0; k < RX_PER; ++k) {
        const int64_t c = (int64_t)blockIdx.x * RX_CH + k * RX_T + threadIdx.x;
        const int f = c < N ? B.flags[c] : 0;
        int tot;
        const int p = pos + block_scan(f, tot, s_w);
        if (f) B.cells[p] = (int)c;
        pos += tot;
    }
}

__global__ void __launch_bounds__(RX_T) mn_hist_kernel(HsLattice L, RelaxBufs B, int pass) {
    __shared__ int s_h[MN_BINS];
    const RelaxState *s = B.st;
    if (s->done || s->mode != 2) return;
    const int lo = c_mn_lo[pass], bits = c_mn_bits[pass];
    const int hi = lo + bits;
    for (int j = threadIdx.x; j < MN_BINS; j += RX_T) s_h[j] = 0;
    __syncthreads();
    const uint64_t prefix = s->prefix, call = s->call;
    const int n = s->count;
    for (int e = blockIdx.x * RX_T + threadIdx.x; e < n; e += gridDim.x * RX_T) {
        const uint64_t key = u53_bits(L.seed, call, (uint32_t)e);
        if ((key >> hi) == prefix) atomicAdd(&s_h[(key >> lo) & ((1u << bits) - 1u)], 1);
    }
    __syncthreads();
    int *g = B.hist + pass * MN_BINS;
    for (int j = threadIdx.x; j < (1 << bits); j += RX_T)
        if (s_h[j]) atomicAdd(&g[j], s_h[j]);
}

__global__ void __launch_bounds__(1024) mn_pick_kernel(RelaxBufs B, int pass) {
    __shared__ int s_c[1024];
    RelaxState *s = B.st;
    if (s->done || s->mode != 2) return;
    const int bits = c_mn_bits[pass];
    const int nb = 1 << bits;
    const int *h = B.hist + pass * MN_BINS;
    const int per = (nb + 1023) / 1024;
    int loc = 0;
    for (int j = 0; j < per; ++j) {
        const int b = threadIdx.x * per + j;
        if (b < nb) loc += h[b];
    }
    s_c[threadIdx.x] = loc;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {      // inclusive scan (Hillis-Steele)
        const int v = (int)threadIdx.x >= o ? s_c[threadIdx.x - o] : 0;
        __syncthreads();
        s_c[threadIdx.x] += v;
        __syncthreads();
    }
    const int k = s->k_rem;
    int cum = threadIdx.x ? s_c[threadIdx.x - 1] : 0;
    if (cum < k && k <= s_c[threadIdx.x]) {   // exactly one thread holds the crossing bin
        for (int j = 0; j < per; ++j) {
            const int b = threadIdx.x * per + j;
            if (b >= nb) break;
            if (cum + h[b] >= k) {
                s->prefix = (s->prefix << bits) | (uint64_t)b;
                s->k_rem = k - cum;
                s->eq_total = h[b];
                break;
            }
            cum += h[b];
        }
    }
}

// Per block: keys below the threshold and keys equal to it.
__global__ void __launch_bounds__(RX_T) mn_select_count_kernel(HsLattice L, RelaxBufs B) {
    __shared__ int s_w[RX_T / 32];
    const RelaxState *s = B.st;
    if (s->done || s->mode != 2) return;
    const uint64_t T = s->prefix, call = s->call;
    const int n = s->count;
    int lt = 0, eq = 0;
#pragma unroll
    for (int k = 0; k < RX_PER; ++k) {
        const int e = blockIdx.x * RX_CH + k * RX_T + threadIdx.x;
        if (e >= n) continue;
        const uint64_t key = u53_bits(L.seed, call, (uint32_t)e);
        lt += key < T;
        eq += key == T;
    }
    lt = block_sum(lt, s_w);
    eq = block_sum(eq, s_w);
    if (threadIdx.x == 0) { B.blk[blockIdx.x] = lt; B.blk2[blockIdx.x] = eq; }
}

// The k chosen cells in list order: every key below the threshold and the first k_rem keys
// equal to it; flips, counters, sublattice counts.
__global__ void __launch_bounds__(RX_T) mn_select_write_kernel(HsLattice L, HsCounters *C, RelaxBufs B,
                                                               HsSwitchList sw) {
    __shared__ int s_w[RX_T / 32];
    __shared__ int s_base[2];
    const RelaxState *s = B.st;
    if (s->done || s->mode != 2) return;
    const uint64_t T = s->prefix, call = s->call;
    const int n = s->count, k_rem = s->k_rem;
    // taken / equal keys in the blocks before this one (a scan over the block counts)
    int taken = 0, eq_run = 0;
    for (int j0 = 0; j0 < (int)blockIdx.x; j0 += RX_T) {
        const int j = j0 + threadIdx.x;
        const int e_here = j < (int)blockIdx.x ? B.blk2[j] : 0;
        int e_tot;
        const int eq_before = eq_run + block_scan(e_here, e_tot, s_w);
        const int t_here = j < (int)blockIdx.x ? B.blk[j] + max(0, min(e_here, k_rem - eq_before)) : 0;
        taken += block_sum(t_here, s_w);
        eq_run += e_tot;
    }
    if (threadIdx.x == 0) {
        s_base[0] = taken;
        s_base[1] = eq_run;
        if (blockIdx.x == 0) {
            C->n_sw = s->k;
            C->switches += s->k;
            C->attempted += s->k;
        }
    }
    __syncthreads();
    int pos = s_base[0], eqb = s_base[1];
#pragma unroll 1
    for (int k = 0; k < RX_PER; ++k) {
        const int e = blockIdx.x * RX_CH + k * RX_T + threadIdx.x;
        uint64_t key = ~0ull;
        if (e < n) key = u53_bits(L.seed, call, (uint32_t)e);
        const int is_eq = e < n && key == T;
        int eq_tot;
        const int eq_rank = eqb + block_scan(is_eq, eq_tot, s_w);
        const int take = e < n && (key < T || (is_eq && eq_rank < k_rem));
        int tot;
        const int p = pos + block_scan(take, tot, s_w);
        if (take) {
            const int c = B.cells[e];
            const int y = c / L.nx, x = c % L.nx;
            sw.y[p] = y;
            sw.x[p] = x;
            L.m[c] = (int8_t)(-L.m[c]);
            L.mm[c] = -L.mm[c];
            atomicAdd(&B.sub_counts[(y % L.uy) * L.ux + (x % L.ux)], 1);
        }
        pos += tot;
        eqb += eq_tot;
    }
}

__global__ void __launch_bounds__(RX_T) mn_mode_kernel(HsLattice L, const HsCounters *C, RelaxBufs B, HsSwitchList sw) {
    const RelaxState *s = B.st;
    if (s->done || s->mode != 2 || !sw.mode) return;
    const int n = C->n_sw;
    for (int j = blockIdx.x * RX_T + threadIdx.x; j < n; j += gridDim.x * RX_T) {
        const int y = sw.y[j], x = sw.x[j];
        sw.mode[j] = B.sub_counts[(y % L.uy) * L.ux + (x % L.ux)] > L.trunc_cutoff ? 1 : 0;
    }
}

// ---------------------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------------------
int64_t n_cells(const HsLattice &L) { return (int64_t)L.nx * L.ny; }
int grid_blocks(const HsLattice &L) { return (int)((n_cells(L) + RX_CH - 1) / RX_CH); }

// One layout serves relax and minimize.
int64_t layout(const HsLattice &L, char *base, RelaxBufs *B) {
    const int64_t N = n_cells(L), nb = grid_blocks(L);
    int64_t off = 0;
    auto take = [&](int64_t bytes) { char *p = base ? base + off : nullptr; off += hs_align_up(bytes, 256); return p; };
    RelaxBufs b;
    b.st = reinterpret_cast<RelaxState *>(take(sizeof(RelaxState)));
    b.order = reinterpret_cast<int32_t *>(take(4LL * RX_MAX_P));
    b.blk = reinterpret_cast<int32_t *>(take(4 * nb));
    b.blk2 = reinterpret_cast<int32_t *>(take(4 * nb));
    b.blk_v = reinterpret_cast<double *>(take(8 * nb));
    b.blk_i = reinterpret_cast<int32_t *>(take(4 * nb));
    b.sub_counts = reinterpret_cast<int32_t *>(take(4LL * RX_MAX_U));
    b.flags = reinterpret_cast<uint8_t *>(take(N));
    b.snap = reinterpret_cast<int8_t *>(take(2 * N));
    b.cells = reinterpret_cast<int32_t *>(take(4 * N));
    b.hist = reinterpret_cast<int32_t *>(take(4LL * MN_PASSES * MN_BINS));
    if (B) *B = b;
    return off;
}

int check_common(const HsLattice &L, const char *who, int64_t bytes) {
    if (L.nx <= 0 || L.ny <= 0 || !L.m || !L.mm || !L.occ) { hs_set_error("%s: empty lattice", who); return HS_EINVAL; }
    if (L.ux * L.uy > RX_MAX_U) { hs_set_error("%s: unit cell larger than %d sites", who, RX_MAX_U); return HS_ERANGE; }
    if (n_cells(L) > (int64_t)INT32_MAX / 2) { hs_set_error("%s: lattice too large", who); return HS_ERANGE; }
    if (bytes < layout(L, nullptr, nullptr)) {
        hs_set_error("%s: scratch %lld < %lld bytes", who, (long long)bytes, (long long)layout(L, nullptr, nullptr));
        return HS_ENOMEM;
    }
    return HS_OK;
}

void steps_of(const HsLattice &L, int simultaneous, int &sx, int &sy) {
    sx = simultaneous ? 1 : 2 * L.ux;
    sy = simultaneous ? 1 : 2 * L.uy;
}

}  // namespace

int64_t hs_relax_scratch(const HsLattice &L) { return layout(L, nullptr, nullptr); }

int hs_relax_begin_impl(const HsLattice &L, void *scratch, int64_t bytes, cudaStream_t st) {
    int rc = check_common(L, "hs_relax_begin", bytes);
    if (rc) return rc;
    RelaxBufs B;
    layout(L, reinterpret_cast<char *>(scratch), &B);
    const int64_t N = n_cells(L);
    if (cudaMemsetAsync(B.st, 0, sizeof(RelaxState), st) != cudaSuccess ||
        cudaMemsetAsync(B.order, 0xff, 4 * RX_MAX_P, st) != cudaSuccess ||                // no order yet
        cudaMemcpyAsync(B.snap, L.m, N, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||   // two sweeps back: m0
        cudaMemsetAsync(B.snap + N, 0, N, st) != cudaSuccess) {                            // before it: zeros
        hs_set_error("hs_relax_begin: %s", cudaGetErrorString(cudaGetLastError()));
        return HS_ECUDA;
    }
    return HS_OK;
}

int hs_relax_permute_impl(const HsLattice &L, HsCounters *C, int simultaneous, void *scratch, int64_t bytes,
                          cudaStream_t st) {
    int rc = check_common(L, "hs_relax_permute", bytes);
    if (rc) return rc;
    RelaxBufs B;
    layout(L, reinterpret_cast<char *>(scratch), &B);
    int sx, sy;
    steps_of(L, simultaneous, sx, sy);
    if (sx > L.nx || sy > L.ny) { hs_set_error("hs_relax_permute: lattice smaller than two unit cells"); return HS_EINVAL; }
    relax_perm_kernel<<<1, 1024, 0, st>>>(L, C, B, sx * sy);
    return hs_check_launch("relax_perm_kernel");
}

int hs_relax_subset_impl(const HsLattice &L, HsCounters *C, const HsSwitchList &sw, int i, int ignore_barrier,
                         int simultaneous, void *scratch, int64_t bytes, cudaStream_t st) {
    int rc = check_common(L, "hs_relax_subset", bytes);
    if (rc) return rc;
    RelaxBufs B;
    layout(L, reinterpret_cast<char *>(scratch), &B);
    int sx, sy;
    steps_of(L, simultaneous, sx, sy);
    if (sx > L.nx || sy > L.ny) { hs_set_error("hs_relax_subset: lattice smaller than two unit cells"); return HS_EINVAL; }
    if (i < 0 || i >= sx * sy) { hs_set_error("hs_relax_subset: subgrid %d of %d", i, sx * sy); return HS_EINVAL; }
    const int64_t Mmax = (int64_t)((L.ny + sy - 1) / sy) * ((L.nx + sx - 1) / sx);
    if (sw.cap < Mmax) { hs_set_error("hs_relax_subset: switch list capacity %d < %lld", sw.cap, (long long)Mmax); return HS_EINVAL; }
    const int nblk = (int)((Mmax + RX_CH - 1) / RX_CH);
    if (simultaneous && cudaMemsetAsync(B.sub_counts, 0, 4 * RX_MAX_U, st) != cudaSuccess) {
        hs_set_error("hs_relax_subset: memset failed");
        return HS_ECUDA;
    }
    relax_decide_kernel<<<nblk, RX_T, 0, st>>>(L, B, i, sx, sy, ignore_barrier, simultaneous);
    if ((rc = hs_check_launch("relax_decide_kernel"))) return rc;
    relax_apply_kernel<<<nblk, RX_T, 0, st>>>(L, C, B, sw, i, sx, sy, simultaneous, nblk);
    if ((rc = hs_check_launch("relax_apply_kernel"))) return rc;
    if (L.has_dipolar) return hs_launch_dipolar_update(L, sw, &C->n_sw, 0, HS_UPDATE_MULTIPLE, C, st);
    return HS_OK;
}

int hs_relax_check_impl(const HsLattice &L, HsCounters *C, int n_max, void *scratch, int64_t bytes, cudaStream_t st) {
    int rc = check_common(L, "hs_relax_check", bytes);
    if (rc) return rc;
    RelaxBufs B;
    layout(L, reinterpret_cast<char *>(scratch), &B);
    const int nb = std::min(grid_blocks(L) * RX_PER, 148 * 8);
    relax_compare_kernel<<<nb, RX_T, 0, st>>>(L, C, B);
    if ((rc = hs_check_launch("relax_compare_kernel"))) return rc;
    relax_end_kernel<<<1, 1, 0, st>>>(C, B, n_max);
    return hs_check_launch("relax_end_kernel");
}

int hs_minimize_begin_impl(const HsLattice &L, void *scratch, int64_t bytes, cudaStream_t st) {
    int rc = check_common(L, "hs_minimize_begin", bytes);
    if (rc) return rc;
    RelaxBufs B;
    layout(L, reinterpret_cast<char *>(scratch), &B);
    if (cudaMemsetAsync(B.st, 0, sizeof(RelaxState), st) != cudaSuccess ||
        cudaMemsetAsync(B.snap, 0, n_cells(L), st) != cudaSuccess) {   // visited counts
        hs_set_error("hs_minimize_begin: memset failed");
        return HS_ECUDA;
    }
    return HS_OK;
}

int hs_minimize_step_impl(const HsLattice &L, HsCounters *C, const HsSwitchList &sw, double frac, void *scratch,
                          int64_t bytes, cudaStream_t st) {
    int rc = check_common(L, "hs_minimize_step", bytes);
    if (rc) return rc;
    if (!(frac > 0.0 && frac <= 1.0)) { hs_set_error("hs_minimize_step: frac must lie in (0, 1]"); return HS_EINVAL; }
    if (sw.cap < n_cells(L)) { hs_set_error("hs_minimize_step: switch list capacity %d < nx*ny", sw.cap); return HS_EINVAL; }
    RelaxBufs B;
    layout(L, reinterpret_cast<char *>(scratch), &B);
    const int nblk = grid_blocks(L);
    const int nh = std::min(nblk * RX_PER, 148 * 8);
    mn_scan_kernel<<<nblk, RX_T, 0, st>>>(L, B);
    if ((rc = hs_check_launch("mn_scan_kernel"))) return rc;
    mn_decide_kernel<<<1, 1024, 0, st>>>(L, C, B, sw, nblk, frac);
    if ((rc = hs_check_launch("mn_decide_kernel"))) return rc;
    mn_compact_kernel<<<nblk, RX_T, 0, st>>>(L, B, nblk);
    if ((rc = hs_check_launch("mn_compact_kernel"))) return rc;
    for (int p = 0; p < MN_PASSES; ++p) {
        mn_hist_kernel<<<nh, RX_T, 0, st>>>(L, B, p);
        if ((rc = hs_check_launch("mn_hist_kernel"))) return rc;
        mn_pick_kernel<<<1, 1024, 0, st>>>(B, p);
        if ((rc = hs_check_launch("mn_pick_kernel"))) return rc;
    }
    mn_select_count_kernel<<<nblk, RX_T, 0, st>>>(L, B);
    if ((rc = hs_check_launch("mn_select_count_kernel"))) return rc;
    mn_select_write_kernel<<<nblk, RX_T, 0, st>>>(L, C, B, sw);
    if ((rc = hs_check_launch("mn_select_write_kernel"))) return rc;
    mn_mode_kernel<<<std::min(nblk, 148), RX_T, 0, st>>>(L, C, B, sw);
    if ((rc = hs_check_launch("mn_mode_kernel"))) return rc;
    if (L.has_dipolar) return hs_launch_dipolar_update(L, sw, &C->n_sw, 0, HS_UPDATE_MULTIPLE, C, st);
    return HS_OK;
}
