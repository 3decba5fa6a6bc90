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

#include "hs_steps.cuh"

namespace {

__global__ void __launch_bounds__(MT) metropolis_kernel(HsLattice L, HsCounters *C, HsSwitchList sw, HsGridPlan P,
                                                        MetroScratch S) {
    metro_step_cta(L, C, sw, P, S);
}

}  // namespace

static void metro_sizes(const HsLattice &L, const HsGridPlan &P, int &cap, int &gsz) { hs_metro_sizes(L, P, cap, gsz); }

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
