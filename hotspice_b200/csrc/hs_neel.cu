// (c) Néel-Arrhenius step (hotspice/core.py:679-709 with E_barrier, core.py:625-656).
//
// The reference draws tau_i ~ Exp(scale_i) for every cell and switches argmin tau. Here the
// same variates (Philox call `rng_call`, element = flat cell index) are compared in the log
// domain, key_i = log E1_i + log scale_i, which never overflows:
//   one channel : log scale_i = (b_i - b_min) beta_i
//   two channels: log scale_i = -log(exp(-(b1_i - b_min) beta_i) + exp(-(b2_i - b_min) beta_i))
// With a uniform temperature the b_min shift is common to all cells and is dropped (one pass);
// otherwise a first pass finds b_min. Each CTA reduces (key, index) with warp shuffles (ties go
// to the smaller index, like numpy.nanargmin); the last CTA to finish (atomic ticket) reduces
// the per-CTA results, evaluates the switching time in FP64 and applies the switch.
#include "hs_steps.cuh"
#include "hs_internal.h"

namespace {

constexpr int NEEL_THREADS = 256;
constexpr int NEEL_MAXB = 148 * 8;

struct NeelScratch {
    HsKeyIdx part[NEEL_MAXB];
    double bpart[NEEL_MAXB];
    unsigned int ticket[4];
};

HS_DEV HsKeyIdx block_kmin(HsKeyIdx v, HsKeyIdx *sm) {
    v = hs_warp_kmin(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sm[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = (lane < (int)(blockDim.x >> 5)) ? sm[lane] : HsKeyIdx{0.0, -1};
        v = hs_warp_kmin(v);
    }
    return v;
}

HS_DEV double block_dmin(double v, double *sm) {
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
    return v;
}

// Returns true when this step must not run (progress() finished); the first kernel of a step
// evaluates the stop rule and records it.
HS_DEV bool neel_stop(const HsLattice &L, HsCounters *C, bool first) {
    if (C->done) return true;
    if (first && !hs_progress_continue(C, L.n_occ)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) { C->done = 1; C->n_sw = 0; }
        return true;
    }
    return false;
}

// Pass 1 (non-uniform temperature only): b_min = nanmin over occupied cells of min(b1, b2).
__global__ void __launch_bounds__(NEEL_THREADS) neel_bmin_kernel(HsLattice L, HsCounters *C, NeelScratch *S) {
    if (neel_stop(L, C, true)) return;
    __shared__ double sm[32];
    __shared__ bool last;
    const int64_t N = (int64_t)L.nx * L.ny;
    double v = INFINITY;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        if (!L.occ[i]) continue;
        double b1, b2;
        hs_barriers(L, (int)(i / L.nx), (int)(i % L.nx), b1, b2);
        v = fmin(v, fmin(b1, b2));
    }
    v = block_dmin(v, sm);
    if (threadIdx.x == 0) {
        S->bpart[blockIdx.x] = v;
        __threadfence();
        last = atomicAdd(&S->ticket[1], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double w = INFINITY;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) w = fmin(w, __ldcg(&S->bpart[b]));
    __syncthreads();
    w = block_dmin(w, sm);
    if (threadIdx.x == 0) { C->bmin = w; S->ticket[1] = 0u; }
}

template <bool TWO, bool UNIF>
__global__ void __launch_bounds__(NEEL_THREADS)
neel_scan_kernel(HsLattice L, HsCounters *C, HsSwitchList sw, double attempt_freq, NeelScratch *S) {
    if (neel_stop(L, C, UNIF)) return;
    __shared__ HsKeyIdx sm[32];
    __shared__ bool last;
    const int64_t N = (int64_t)L.nx * L.ny;
    const uint64_t call = C->rng_call;
    const double bmin = UNIF ? 0.0 : C->bmin;
    HsKeyIdx best = neel_scan_range(L, blockIdx.x * (int64_t)blockDim.x + threadIdx.x, (int64_t)gridDim.x * blockDim.x,
                                    N, call, bmin, HsKeyIdx{0.0, -1});
    best = block_kmin(best, sm);
    if (threadIdx.x == 0) {
        S->part[blockIdx.x] = best;
        __threadfence();
        last = atomicAdd(&S->ticket[0], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    HsKeyIdx w{0.0, -1};
    for (int b = threadIdx.x; b < (int)gridDim.x; b += blockDim.x) {
        HsKeyIdx p;
        p.key = __ldcg(&S->part[b].key);
        p.idx = __ldcg(&S->part[b].idx);
        p.b1 = __ldcg(&S->part[b].b1);
        p.b2 = __ldcg(&S->part[b].b2);
        p.mm = __ldcg(&S->part[b].mm);
        p.m = __ldcg(&S->part[b].m);
        w = hs_kmin(w, p);
    }
    __syncthreads();
    w = block_kmin(w, sm);
    if (threadIdx.x != 0) return;
    S->ticket[0] = 0u;
    neel_finalize(L, C, sw, w, call, bmin, UNIF, TWO, attempt_freq);
}

}  // namespace

// The engine keeps its barrier cache (one float per cell) behind the step's own scratch.
static_assert(sizeof(NeelScratch) <= HS_NEEL_CACHE_OFFSET, "Néel scratch overlaps the barrier cache");
int64_t hs_neel_scratch(const HsLattice &L) { return HS_NEEL_CACHE_OFFSET + 4 * (int64_t)L.nx * L.ny; }

int hs_launch_neel(const HsLattice &L, HsCounters *C, const HsSwitchList &sw, double attempt_freq,
                   void *scratch, int64_t scratch_bytes, cudaStream_t st) {
    if (scratch_bytes < (int64_t)sizeof(NeelScratch)) {
        hs_set_error("hs_neel_step: scratch %lld < %lld bytes", (long long)scratch_bytes, (long long)sizeof(NeelScratch));
        return HS_ENOMEM;
    }
    if (sw.cap < 1) { hs_set_error("hs_neel_step: switch list capacity < 1"); return HS_EINVAL; }
    NeelScratch *S = reinterpret_cast<NeelScratch *>(scratch);
    const int64_t N = (int64_t)L.nx * L.ny;
    const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((N + NEEL_THREADS - 1) / NEEL_THREADS, NEEL_MAXB));
    const bool unif = L.beta_uniform > 0.0;
    const bool two = L.use_perp != 0;
    if (!unif) neel_bmin_kernel<<<blocks, NEEL_THREADS, 0, st>>>(L, C, S);
    if (two) {
        if (unif) neel_scan_kernel<true, true><<<blocks, NEEL_THREADS, 0, st>>>(L, C, sw, attempt_freq, S);
        else neel_scan_kernel<true, false><<<blocks, NEEL_THREADS, 0, st>>>(L, C, sw, attempt_freq, S);
    } else {
        if (unif) neel_scan_kernel<false, true><<<blocks, NEEL_THREADS, 0, st>>>(L, C, sw, attempt_freq, S);
        else neel_scan_kernel<false, false><<<blocks, NEEL_THREADS, 0, st>>>(L, C, sw, attempt_freq, S);
    }
    int rc = hs_check_launch("neel_scan_kernel");
    if (rc) return rc;
    if (L.has_dipolar) return hs_launch_dipolar_update(L, sw, &C->n_sw, 0, HS_UPDATE_SINGLE, C, st);
    return HS_OK;
}
