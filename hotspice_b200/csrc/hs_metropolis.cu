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
                                                        MetroScratch S, int ws_bytes) {
    extern __shared__ __align__(16) unsigned char s_ws[];   // the Poisson-disc sampler's arrays, if given
    metro_step_cta(L, C, sw, P, S, ws_bytes > 0 ? s_ws : nullptr, ws_bytes);
}

constexpr int64_t METRO_WS_MAX = 200 * 1024;   // dynamic shared memory the Poisson sampler may use

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
    int ws = 0;
    if (P.sample_scheme == HS_SAMPLE_POISSON && hs_poisson_mem_bytes(gsz) <= METRO_WS_MAX) {
        ws = (int)hs_poisson_mem_bytes(gsz);
        static int granted = 0;
        if (ws > 48 * 1024 && ws > granted) {
            cudaError_t e = cudaFuncSetAttribute(metropolis_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)METRO_WS_MAX);
            if (e != cudaSuccess) { hs_set_error("metropolis_kernel: %s", cudaGetErrorString(e)); return HS_ECUDA; }
            granted = (int)METRO_WS_MAX;
        }
    }
    metropolis_kernel<<<1, MT, ws, st>>>(L, C, sw, P, S, ws);
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
// address with cudaGetSymbolAddress; make that first call before any stream capture. The
// address is kept with the id of the device's context: after a cudaDeviceReset (a new
// primary context) the next call looks it up again, so that call too must come before any
// capture. Every call shares the array and it keeps the previous call's contents: the kernel
// rewrites every entry it reads (nothing has to start at zero), and calls that overlap on the
// GPU (other streams, other threads) race on it.
// ---------------------------------------------------------------------------------------
#include <cuda.h>   // types of the two driver entry points below (resolved at run time)
#include <mutex>

#define HS_NOALLOC_METRO_BYTES (4LL << 20)   // 4 MiB
#define HS_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) unsigned char g_hs_metro_scratch[HS_NOALLOC_METRO_BYTES];

namespace {
struct NoallocSlot { void *ptr; unsigned long long ctx_id; };
NoallocSlot g_noalloc[HS_NOALLOC_MAX_DEVICES];
std::mutex g_noalloc_mu;
typedef CUresult (*PfnCtxGetCurrent)(CUcontext *);
typedef CUresult (*PfnCtxGetId)(CUcontext, unsigned long long *);
PfnCtxGetCurrent g_ctx_current = nullptr;
PfnCtxGetId g_ctx_id = nullptr;

// Id of the calling thread's current context (0 when there is none or it cannot be read).
unsigned long long current_ctx_id() {
    if (!g_ctx_current) {
        cudaDriverEntryPointQueryResult q1, q2;
        void *f1 = nullptr, *f2 = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
            cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) != cudaSuccess || !f1 || !f2)
            return 0;
        g_ctx_id = reinterpret_cast<PfnCtxGetId>(f2);
        g_ctx_current = reinterpret_cast<PfnCtxGetCurrent>(f1);
    }
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (g_ctx_current(&c) != CUDA_SUCCESS || !c || g_ctx_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}
}  // namespace

extern "C" int hs_metropolis_step_noalloc(const HsLattice *L, HsCounters *C, const HsSwitchList *sw,
                                          const HsGridPlan *P, void *stream) {
    // every argument check before anything is sized or looked up
    int rc = hs_check_metropolis_args(L, C, sw, P, "hs_metropolis_step_noalloc");
    if (rc) return rc;
    const int64_t need = hs_metropolis_scratch(*L, *P);
    if (need > HS_NOALLOC_METRO_BYTES) {
        hs_set_error("hs_metropolis_step_noalloc: this selection plan needs %lld bytes of scratch, the fixed "
                     "scratch holds %lld; use hs_metropolis_step with a caller-provided buffer",
                     (long long)need, (long long)HS_NOALLOC_METRO_BYTES);
        return HS_ERANGE;
    }
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) { hs_set_error("hs_metropolis_step_noalloc: cudaGetDevice: %s", cudaGetErrorString(e)); return HS_ECUDA; }
    if (dev < 0 || dev >= HS_NOALLOC_MAX_DEVICES) {
        hs_set_error("hs_metropolis_step_noalloc: device %d beyond the %d supported", dev, HS_NOALLOC_MAX_DEVICES);
        return HS_ERANGE;
    }
    void *ptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        NoallocSlot &slot = g_noalloc[dev];
        const unsigned long long id = current_ctx_id();
        if (!slot.ptr || id == 0 || id != slot.ctx_id) {  // set-up: once per device (and per context)
            ptr = nullptr;
            e = cudaGetSymbolAddress(&ptr, g_hs_metro_scratch);
            if (e != cudaSuccess || !ptr) {
                hs_set_error("hs_metropolis_step_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
                return HS_ECUDA;
            }
            slot.ptr = ptr;
            slot.ctx_id = current_ctx_id();   // the look-up made the device's context current
        }
        ptr = slot.ptr;
    }
    return hs_metropolis_step(L, C, sw, P, ptr, HS_NOALLOC_METRO_BYTES, stream);
}
