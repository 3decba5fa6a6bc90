// Packed host <-> device state transfer for batches of instances.
//
// A batch's per-instance arrays (spins, m * moment, counters, energies) live in separate device
// allocations. Moving them one cudaMemcpyAsync at a time costs a host call per array (thousands
// per launch for a large batch). Instead the caller packs them into one staging buffer, moves
// it with ONE copy, and this kernel scatters the staging buffer into the arrays (or gathers the
// arrays into it) from a device table of segments: {offset in the staging buffer, device
// address, bytes}, each at most HS_SEGMENT_MAX bytes, one CTA per segment (grid-stride).
// Both addresses of a segment are 16-byte aligned except possibly at its tail, which is copied
// byte by byte.
#include "hs_common.cuh"
#include "hs_internal.h"

namespace {

constexpr int SG_T = 256;

__global__ void __launch_bounds__(SG_T) segments_kernel(char *staged, const HsSegment *segs, int n, int to_device) {
    for (int s = blockIdx.x; s < n; s += gridDim.x) {
        const HsSegment g = segs[s];
        char *a = staged + g.staged;                       // staging side
        char *b = reinterpret_cast<char *>(g.device);      // array side
        const char *src = to_device ? a : b;
        char *dst = to_device ? b : a;
        const int64_t nv = ((reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) & 15) ? 0 : g.bytes / 16;
        const int4 *s4 = reinterpret_cast<const int4 *>(src);
        int4 *d4 = reinterpret_cast<int4 *>(dst);
        for (int64_t k = threadIdx.x; k < nv; k += SG_T) d4[k] = s4[k];
        for (int64_t k = nv * 16 + threadIdx.x; k < g.bytes; k += SG_T) dst[k] = src[k];
    }
}

}  // namespace

int hs_segments_copy_impl(void *staged, const HsSegment *segs, int n, int to_device, cudaStream_t st) {
    const int blocks = std::min(n, 148 * 16);
    segments_kernel<<<blocks, SG_T, 0, st>>>(reinterpret_cast<char *>(staged), segs, n, to_device);
    return hs_check_launch("segments_kernel");
}
