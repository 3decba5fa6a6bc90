// (e) Wolff cluster step for exchange-only lattices (hotspice/core.py:588-602, 711-718).
//
// The reference grows the cluster layer by layer: frontier = (1 - checked) * conv(cluster, NN),
// every frontier cell is marked checked, accepted with probability 1 - exp(-2 J / kBT * count)
// (one full-grid uniform draw per layer), and the accepted cells join the cluster.
// Cells adjacent to an older cluster cell were already checked one layer after that cell
// joined, so the frontier of layer L is exactly the unchecked neighbours (same spin as the
// seed) of the cells added in layer L-1. This kernel therefore keeps the BFS sparse: only
// those cells are visited and only their variates are evaluated (element = flat cell index of
// the layer's Philox call, so the decisions are the reference's). Membership bookkeeping uses
// per-cell epoch stamps, so nothing has to be cleared between clusters. Integer decisions
// against FP64 thresholds: bit-exact with the reference given the same variates.
#include "hs_common.cuh"
#include "hs_internal.h"

#include "hs_steps.cuh"

namespace {

__global__ void __launch_bounds__(WT) wolff_kernel(HsLattice L, HsCounters *C, HsSwitchList sw, WolffScratch S) {
    wolff_step_cta(L, C, sw, S);
}

}  // namespace

int64_t hs_wolff_scratch(const HsLattice &L) {
    const int64_t N = (int64_t)L.nx * L.ny;
    return 5 * hs_align_up(4 * N, 256) + 256;     // + the stamp epoch
}

int hs_launch_wolff(const HsLattice &L, HsCounters *C, const HsSwitchList &sw, void *scratch, int64_t scratch_bytes,
                    cudaStream_t st) {
    if (!L.has_exchange || L.has_dipolar) {
        hs_set_error("hs_wolff_step: Wolff clusters need an exchange-only system (core.py:577-590)");
        return HS_EINVAL;
    }
    if (scratch_bytes < hs_wolff_scratch(L)) {
        hs_set_error("hs_wolff_step: scratch %lld < %lld bytes", (long long)scratch_bytes, (long long)hs_wolff_scratch(L));
        return HS_ENOMEM;
    }
    const int64_t N = (int64_t)L.nx * L.ny;
    char *p = reinterpret_cast<char *>(scratch);
    WolffScratch S;
    S.chk_ep = reinterpret_cast<int32_t *>(p); p += hs_align_up(4 * N, 256);
    S.cl_ep = reinterpret_cast<int32_t *>(p); p += hs_align_up(4 * N, 256);
    S.cl_layer = reinterpret_cast<int32_t *>(p); p += hs_align_up(4 * N, 256);
    S.list = reinterpret_cast<int32_t *>(p); p += hs_align_up(4 * N, 256);
    S.cand = reinterpret_cast<int32_t *>(p); p += hs_align_up(4 * N, 256);
    S.epoch = reinterpret_cast<int32_t *>(p);
    wolff_kernel<<<1, WT, 0, st>>>(L, C, sw, S);
    return hs_check_launch("wolff_kernel");
}
