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

namespace {

constexpr int WT = 1024;

struct WolffScratch {
    int32_t *chk_ep;   // epoch in which the cell was checked (seed or frontier)
    int32_t *cl_ep;    // epoch in which the cell joined the cluster
    int32_t *cl_layer; // layer in which it joined
    int32_t *list;     // cluster cells in BFS order (capacity N)
    int32_t *cand;     // frontier of the current layer (capacity N)
};

__global__ void __launch_bounds__(WT) wolff_kernel(HsLattice L, HsCounters *C, HsSwitchList sw, WolffScratch S) {
    __shared__ int s_ncand, s_nacc, s_epoch;
    if (C->done) return;
    if (!hs_progress_continue(C, L.n_occ)) {
        if (threadIdx.x == 0) { C->done = 1; C->n_sw = 0; }
        return;
    }
    const int nx = L.nx, ny = L.ny;
    const int64_t N = (int64_t)nx * ny;
    uint64_t call = C->rng_call;
    if (threadIdx.x == 0) { s_epoch = C->epoch + 1; C->epoch = s_epoch; }
    // seed: _select_single (np.random.randint(n) -> nonzero index)
    const int seed = L.nonzero[(int)floor(hs_u53(L.seed, call, 0u) * L.n_occ)];
    call += 1;
    __syncthreads();
    const int epoch = s_epoch;
    const int8_t ms = L.m[seed];
    if (threadIdx.x == 0) {
        S.chk_ep[seed] = epoch;
        S.cl_ep[seed] = epoch;
        S.cl_layer[seed] = 0;
        S.list[0] = seed;
    }
    int lstart = 0, lend = 1;
    const int ch = L.nn_h / 2, cw = L.nn_w / 2;
    const double m2J = -2.0 * L.J;
    int layer = 1;
    for (; layer <= (int)N + 1; ++layer) {
        if (threadIdx.x == 0) { s_ncand = 0; s_nacc = 0; }
        __syncthreads();
        // frontier: unchecked same-spin cells j with q = j + c - b for a new cell q, mask[b] != 0
        for (int t = lstart + threadIdx.x; t < lend; t += blockDim.x) {
            const int q = S.list[t];
            const int qy = q / nx, qx = q % nx;
            for (int a = 0; a < L.nn_h; ++a)
                for (int b = 0; b < L.nn_w; ++b) {
                    if (!L.nn[a * L.nn_w + b]) continue;
                    int jy = qy - ch + a, jx = qx - cw + b;
                    if (L.pbc) { jy = hs_wrap(jy, ny); jx = hs_wrap(jx, nx); }
                    else if (jy < 0 || jy >= ny || jx < 0 || jx >= nx) continue;
                    const int j = jy * nx + jx;
                    if (L.m[j] != ms) continue;
                    if (atomicExch(&S.chk_ep[j], epoch) == epoch) continue;
                    S.cand[atomicAdd(&s_ncand, 1)] = j;
                }
        }
        __syncthreads();
        const int ncand = s_ncand;
        if (ncand == 0) break;  // empty frontier: the reference's while-loop ends, no draw
        for (int t = threadIdx.x; t < ncand; t += blockDim.x) {
            const int j = S.cand[t];
            const int jy = j / nx, jx = j % nx;
            int count = 0;
            for (int a = 0; a < L.nn_h; ++a)
                for (int b = 0; b < L.nn_w; ++b) {
                    const int w = L.nn[a * L.nn_w + b];
                    if (!w) continue;
                    int yy = jy + ch - a, xx = jx + cw - b;
                    if (L.pbc) { yy = hs_wrap(yy, ny); xx = hs_wrap(xx, nx); }
                    else if (yy < 0 || yy >= ny || xx < 0 || xx >= nx) continue;
                    const int k = yy * nx + xx;
                    if (S.cl_ep[k] == epoch && S.cl_layer[k] < layer) count += w;
                }
            // bond = 1 - exp(-2 J / kBT * count), kBT = 1/beta (hotspice/core.py:599)
            double bond;
            if (L.wolff_bond && count <= 24) {
                bond = L.wolff_bond[count];
            } else {
                const double kBT = 1.0 / hs_beta(L, j);
                bond = 1.0 - exp(m2J / kBT * (double)count);
            }
            const double u = hs_u53(L.seed, call, (uint32_t)j);
            if (!(u > bond)) {
                S.cl_ep[j] = epoch;
                S.cl_layer[j] = layer;
                S.list[lend + atomicAdd(&s_nacc, 1)] = j;
            }
        }
        call += 1;
        __syncthreads();
        lstart = lend;
        lend += s_nacc;
    }
    if (layer > (int)N + 1 && threadIdx.x == 0) C->status |= HS_ST_WOLFF_OVERFLOW;
    // flip the cluster; counters as in core.py:714-716
    for (int t = threadIdx.x; t < lend; t += blockDim.x) {
        const int j = S.list[t];
        L.m[j] = (int8_t)(-L.m[j]);
        L.mm[j] = -L.mm[j];
        if (t < sw.cap) { sw.y[t] = j / nx; sw.x[t] = j % nx; if (sw.mode) sw.mode[t] = 0; }
    }
    if (threadIdx.x == 0) {
        C->attempted += lend;
        C->switches += lend;
        C->rng_call = call;
        C->n_sw = min(lend, sw.cap);
        C->steps += 1;
        if (lend > sw.cap) C->status |= HS_ST_SWITCH_OVERFLOW;
    }
}

}  // namespace

int64_t hs_wolff_scratch(const HsLattice &L) {
    const int64_t N = (int64_t)L.nx * L.ny;
    return 5 * hs_align_up(4 * N, 256);
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
    S.cand = reinterpret_cast<int32_t *>(p);
    wolff_kernel<<<1, WT, 0, st>>>(L, C, sw, S);
    return hs_check_launch("wolff_kernel");
}
