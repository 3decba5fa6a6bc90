// extern "C" entry points of libhotspice_sm100.so (declared in include/hotspice_b200.h).
#include <cstdarg>
#include <cstdio>
#include <cstring>

#include "hs_common.cuh"
#include "hs_internal.h"

namespace {
thread_local char g_err[512] = "";

__global__ void philox_kernel(uint64_t seed, uint64_t call, int32_t n, double *out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        out[i] = hs_u53(seed, call, (uint32_t)i);
}

__global__ void exchange_energy_kernel(HsLattice L, float *E, float *Ep) {
    const int64_t N = (int64_t)L.nx * L.ny;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        double e, ep;
        hs_exchange_at(L, (int)(i / L.nx), (int)(i % L.nx), e, ep);
        E[i] = (float)e;
        if (Ep) Ep[i] = (float)ep;
    }
}

__global__ void switch_energy_kernel(HsLattice L, float *dE) {
    const int64_t N = (int64_t)L.nx * L.ny;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
        double e, ep;
        hs_energy_at(L, (int)(i / L.nx), (int)(i % L.nx), e, ep);
        dE[i] = (float)(-2.0 * e);
    }
}

int grid_for(int64_t n, int threads) {
    return (int)std::max<int64_t>(1, std::min<int64_t>((n + threads - 1) / threads, 148 * 16));
}

int check_lattice(const HsLattice *L, const char *who) {
    if (!L) { hs_set_error("%s: null lattice", who); return HS_EINVAL; }
    if (L->nx <= 0 || L->ny <= 0 || L->ux <= 0 || L->uy <= 0) { hs_set_error("%s: bad lattice size", who); return HS_EINVAL; }
    if ((int64_t)L->nx * L->ny >= (1LL << 31)) { hs_set_error("%s: lattice larger than 2^31 cells", who); return HS_ERANGE; }
    if (!L->m || !L->occ || !L->mm || !L->E_B) { hs_set_error("%s: missing state array", who); return HS_EINVAL; }
    if (L->has_dipolar && (!L->K || !L->E_dip || !L->sub_of)) { hs_set_error("%s: missing dipolar arrays", who); return HS_EINVAL; }
    if (L->has_dipolar && L->use_perp && (!L->Kpo || !L->E_dip_perp)) { hs_set_error("%s: missing perp arrays", who); return HS_EINVAL; }
    if (L->has_exchange && (L->nn_h * L->nn_w > 28 || L->nn_h % 2 == 0 || L->nn_w % 2 == 0)) {
        hs_set_error("%s: exchange mask must be odd-sized and at most 28 cells", who); return HS_EINVAL;
    }
    if (L->has_exchange && L->in_plane && !L->orient) { hs_set_error("%s: in-plane exchange needs orientation", who); return HS_EINVAL; }
    if (L->beta_uniform <= 0.0 && !L->beta) { hs_set_error("%s: missing beta", who); return HS_EINVAL; }
    if (L->n_occ <= 0 || !L->nonzero) { hs_set_error("%s: lattice has no magnets", who); return HS_EINVAL; }
    return HS_OK;
}
}  // namespace

int hs_check_metropolis_plan(const HsLattice *L, const HsGridPlan *P, const char *who) {
    int rc = check_lattice(L, who);
    if (rc) return rc;
    if (!P) { hs_set_error("%s: null plan", who); return HS_EINVAL; }
    if (P->sample_scheme == HS_SAMPLE_GRID && (!P->phase_off || !P->phase_yx || P->Rx < 1 || P->Ry < 1 || P->n_sc < 1)) {
        hs_set_error("%s: bad grid plan", who); return HS_EINVAL;
    }
    if (P->sample_scheme == HS_SAMPLE_POISSON) {
        if (!(P->r_cells >= 0.0) || !(P->r_cells < 1e9)) { hs_set_error("%s: bad Poisson radius", who); return HS_EINVAL; }
        if (hs_poisson_grid_cells(*L, *P) > HS_POISSON_GRID_MAX) {
            hs_set_error("%s: Poisson-disc background grid of %.0f cells exceeds %d", who, hs_poisson_grid_cells(*L, *P),
                         HS_POISSON_GRID_MAX);
            return HS_ERANGE;
        }
    }
    if (P->sample_scheme != HS_SAMPLE_GRID && P->sample_scheme != HS_SAMPLE_POISSON && P->sample_scheme != HS_SAMPLE_SINGLE) {
        hs_set_error("%s: unknown sample scheme %d", who, P->sample_scheme); return HS_EINVAL;
    }
    return HS_OK;
}

int hs_check_metropolis_args(const HsLattice *L, const HsCounters *C, const HsSwitchList *sw, const HsGridPlan *P,
                             const char *who) {
    int rc = hs_check_metropolis_plan(L, P, who);
    if (rc) return rc;
    if (!C || !sw) { hs_set_error("%s: null argument", who); return HS_EINVAL; }
    return HS_OK;
}

void hs_set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int hs_check_launch(const char *what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        hs_set_error("%s: %s", what, cudaGetErrorString(e));
        return HS_ECUDA;
    }
    return HS_OK;
}

int hs_launch_philox(uint64_t seed, uint64_t call, int32_t n, double *out, cudaStream_t st) {
    philox_kernel<<<grid_for(n, 256), 256, 0, st>>>(seed, call, n, out);
    return hs_check_launch("philox_kernel");
}

int hs_launch_exchange_energy(const HsLattice &L, float *E, float *Ep, cudaStream_t st) {
    exchange_energy_kernel<<<grid_for((int64_t)L.nx * L.ny, 256), 256, 0, st>>>(L, E, Ep);
    return hs_check_launch("exchange_energy_kernel");
}

int hs_launch_switch_energy(const HsLattice &L, float *dE, cudaStream_t st) {
    switch_energy_kernel<<<grid_for((int64_t)L.nx * L.ny, 256), 256, 0, st>>>(L, dE);
    return hs_check_launch("switch_energy_kernel");
}

extern "C" {

int hs_version(void) { return 1; }

int hs_last_error(char *buf, int len) {
    if (!buf || len <= 0) return HS_EINVAL;
    strncpy(buf, g_err, (size_t)len - 1);
    buf[len - 1] = '\0';
    return HS_OK;
}

int hs_struct_sizes(int32_t *out, int n) {
    const int32_t s[7] = {(int32_t)sizeof(HsLattice), (int32_t)sizeof(HsCounters), (int32_t)sizeof(HsSwitchList),
                          (int32_t)sizeof(HsGridPlan), (int32_t)offsetof(HsLattice, nx), (int32_t)sizeof(HsInstance),
                          (int32_t)sizeof(HsSegment)};
    for (int i = 0; i < n && i < 7; ++i) out[i] = s[i];
    return HS_OK;
}

int hs_philox_uniform(uint64_t seed, uint64_t call, int32_t n, double *out, void *stream) {
    if (n < 0 || (n > 0 && !out)) { hs_set_error("hs_philox_uniform: bad arguments"); return HS_EINVAL; }
    if (n == 0) return HS_OK;
    return hs_launch_philox(seed, call, n, out, (cudaStream_t)stream);
}

int hs_dipolar_update(const HsLattice *L, const HsSwitchList *sw, const int32_t *n_sw_dev, int32_t n_host,
                      int32_t semantics, const HsCounters *C, void *stream) {
    int rc = check_lattice(L, "hs_dipolar_update");
    if (rc) return rc;
    if (!L->has_dipolar) { hs_set_error("hs_dipolar_update: lattice has no dipolar energy"); return HS_EINVAL; }
    if (!sw || (!n_sw_dev && n_host < 0) || (n_host > sw->cap && !n_sw_dev)) {
        hs_set_error("hs_dipolar_update: bad switch list"); return HS_EINVAL;
    }
    if (semantics != HS_UPDATE_SINGLE && semantics != HS_UPDATE_MULTIPLE) {
        hs_set_error("hs_dipolar_update: bad semantics"); return HS_EINVAL;
    }
    if (!n_sw_dev && n_host == 0) return HS_OK;
    return hs_launch_dipolar_update(*L, *sw, n_sw_dev, n_host, semantics, C, (cudaStream_t)stream);
}

int hs_dipolar_full_direct(const HsLattice *L, int32_t fp64, double *E64, double *Ep64, void *stream) {
    int rc = check_lattice(L, "hs_dipolar_full_direct");
    if (rc) return rc;
    if (!L->has_dipolar) { hs_set_error("hs_dipolar_full_direct: lattice has no dipolar energy"); return HS_EINVAL; }
    if (L->use_perp && !L->Kps) { hs_set_error("hs_dipolar_full_direct: missing perp-self kernels"); return HS_EINVAL; }
    if (fp64 && (!E64 || (L->use_perp && !Ep64))) { hs_set_error("hs_dipolar_full_direct: missing FP64 outputs"); return HS_EINVAL; }
    return hs_launch_dipolar_full_direct(*L, fp64, E64, Ep64, (cudaStream_t)stream);
}

int64_t hs_igemm_scratch_bytes(const HsLattice *L, int32_t nsplit) {
    if (check_lattice(L, "hs_igemm_scratch_bytes")) return -1;
    return hs_igemm_scratch(*L, nsplit);
}

int hs_dipolar_full_igemm(const HsLattice *L, int32_t nsplit, void *scratch, int64_t scratch_bytes, void *stream) {
    int rc = check_lattice(L, "hs_dipolar_full_igemm");
    if (rc) return rc;
    if (!L->has_dipolar) { hs_set_error("hs_dipolar_full_igemm: lattice has no dipolar energy"); return HS_EINVAL; }
    return hs_launch_igemm(*L, nsplit, scratch, scratch_bytes, (cudaStream_t)stream);
}

int hs_set_wait_limit(uint64_t ns) { return hs_set_wait_limit_impl(ns); }

int64_t hs_neel_scratch_bytes(const HsLattice *L) {
    if (check_lattice(L, "hs_neel_scratch_bytes")) return -1;
    return hs_neel_scratch(*L);
}

int hs_neel_step(const HsLattice *L, HsCounters *C, const HsSwitchList *sw, double attempt_freq, void *scratch,
                 int64_t scratch_bytes, void *stream) {
    int rc = check_lattice(L, "hs_neel_step");
    if (rc) return rc;
    if (!C || !sw || !scratch) { hs_set_error("hs_neel_step: null argument"); return HS_EINVAL; }
    if (!(attempt_freq > 0.0)) { hs_set_error("hs_neel_step: attempt_freq must be > 0"); return HS_EINVAL; }
    return hs_launch_neel(*L, C, *sw, attempt_freq, scratch, scratch_bytes, (cudaStream_t)stream);
}

int64_t hs_metropolis_scratch_bytes(const HsLattice *L, const HsGridPlan *P) {
    if (hs_check_metropolis_plan(L, P, "hs_metropolis_scratch_bytes")) return -1;
    return hs_metropolis_scratch(*L, *P);
}

int hs_metropolis_step(const HsLattice *L, HsCounters *C, const HsSwitchList *sw, const HsGridPlan *P, void *scratch,
                       int64_t scratch_bytes, void *stream) {
    int rc = hs_check_metropolis_args(L, C, sw, P, "hs_metropolis_step");
    if (rc) return rc;
    if (!scratch) { hs_set_error("hs_metropolis_step: null scratch"); return HS_EINVAL; }
    return hs_launch_metropolis(*L, C, *sw, *P, scratch, scratch_bytes, (cudaStream_t)stream);
}

int64_t hs_wolff_scratch_bytes(const HsLattice *L) {
    if (check_lattice(L, "hs_wolff_scratch_bytes")) return -1;
    return hs_wolff_scratch(*L);
}

int hs_wolff_step(const HsLattice *L, HsCounters *C, const HsSwitchList *sw, void *scratch, int64_t scratch_bytes,
                  void *stream) {
    int rc = check_lattice(L, "hs_wolff_step");
    if (rc) return rc;
    if (!C || !sw || !scratch) { hs_set_error("hs_wolff_step: null argument"); return HS_EINVAL; }
    return hs_launch_wolff(*L, C, *sw, scratch, scratch_bytes, (cudaStream_t)stream);
}

int64_t hs_relax_scratch_bytes(const HsLattice *L) {
    if (check_lattice(L, "hs_relax_scratch_bytes")) return -1;
    return hs_relax_scratch(*L);
}

int hs_relax_begin(const HsLattice *L, void *scratch, int64_t scratch_bytes, void *stream) {
    int rc = check_lattice(L, "hs_relax_begin");
    if (rc) return rc;
    if (!scratch) { hs_set_error("hs_relax_begin: null scratch"); return HS_EINVAL; }
    return hs_relax_begin_impl(*L, scratch, scratch_bytes, (cudaStream_t)stream);
}

int hs_relax_permute(const HsLattice *L, HsCounters *C, int32_t simultaneous, void *scratch, int64_t scratch_bytes,
                     void *stream) {
    int rc = check_lattice(L, "hs_relax_permute");
    if (rc) return rc;
    if (!C || !scratch) { hs_set_error("hs_relax_permute: null argument"); return HS_EINVAL; }
    return hs_relax_permute_impl(*L, C, simultaneous, scratch, scratch_bytes, (cudaStream_t)stream);
}

int hs_relax_subset(const HsLattice *L, HsCounters *C, const HsSwitchList *sw, int32_t i, int32_t ignore_barrier,
                    int32_t simultaneous, void *scratch, int64_t scratch_bytes, void *stream) {
    int rc = check_lattice(L, "hs_relax_subset");
    if (rc) return rc;
    if (!C || !sw || !scratch) { hs_set_error("hs_relax_subset: null argument"); return HS_EINVAL; }
    return hs_relax_subset_impl(*L, C, *sw, i, ignore_barrier, simultaneous, scratch, scratch_bytes,
                                (cudaStream_t)stream);
}

int hs_minimize_all(const HsLattice *L, HsCounters *C, const HsSwitchList *sw, int32_t ignore_barrier,
                    int32_t simultaneous, void *scratch, int64_t scratch_bytes, void *stream) {
    int rc = hs_relax_permute(L, C, simultaneous, scratch, scratch_bytes, stream);
    if (rc) return rc;
    const int P = simultaneous ? 1 : 4 * L->ux * L->uy;
    for (int i = 0; i < P; ++i) {
        rc = hs_relax_subset(L, C, sw, i, ignore_barrier, simultaneous, scratch, scratch_bytes, stream);
        if (rc) return rc;
    }
    return HS_OK;
}

int hs_relax_check(const HsLattice *L, HsCounters *C, int32_t n_max, void *scratch, int64_t scratch_bytes,
                   void *stream) {
    int rc = check_lattice(L, "hs_relax_check");
    if (rc) return rc;
    if (!C || !scratch || n_max < 1) { hs_set_error("hs_relax_check: bad argument"); return HS_EINVAL; }
    return hs_relax_check_impl(*L, C, n_max, scratch, scratch_bytes, (cudaStream_t)stream);
}

int hs_minimize_begin(const HsLattice *L, void *scratch, int64_t scratch_bytes, void *stream) {
    int rc = check_lattice(L, "hs_minimize_begin");
    if (rc) return rc;
    if (!scratch) { hs_set_error("hs_minimize_begin: null scratch"); return HS_EINVAL; }
    return hs_minimize_begin_impl(*L, scratch, scratch_bytes, (cudaStream_t)stream);
}

int hs_minimize_step(const HsLattice *L, HsCounters *C, const HsSwitchList *sw, double frac, void *scratch,
                     int64_t scratch_bytes, void *stream) {
    int rc = check_lattice(L, "hs_minimize_step");
    if (rc) return rc;
    if (!C || !sw || !scratch) { hs_set_error("hs_minimize_step: null argument"); return HS_EINVAL; }
    return hs_minimize_step_impl(*L, C, *sw, frac, scratch, scratch_bytes, (cudaStream_t)stream);
}

int hs_zeeman_set(int64_t n_cells, int32_t in_plane, const double *moment, const double *orient, const float *pattern,
                  double magnitude, double angle, double *E_factor, double *E_factor_perp, float *zee, float *zee_perp,
                  void *stream) {
    if (n_cells <= 0 || !moment || !zee || (in_plane && !orient)) { hs_set_error("hs_zeeman_set: bad arguments"); return HS_EINVAL; }
    return hs_zeeman_set_impl(n_cells, in_plane, moment, orient, pattern, magnitude, angle, E_factor, E_factor_perp, zee,
                              zee_perp, (cudaStream_t)stream);
}

int hs_progress_arm(HsCounters *C, int32_t n_occ, double t_max, double MCsteps_max, void *stream) {
    if (!C || n_occ <= 0) { hs_set_error("hs_progress_arm: bad arguments"); return HS_EINVAL; }
    if (!(t_max < INFINITY) && !(MCsteps_max < INFINITY)) {
        hs_set_error("hs_progress_arm: t_max and MCsteps_max are both infinite (the run would never end)");
        return HS_EINVAL;
    }
    return hs_progress_arm_impl(C, n_occ, t_max, MCsteps_max, (cudaStream_t)stream);
}

int hs_square_vertex_counts(const int8_t *m, int32_t nx, int32_t ny, int64_t *out, void *stream) {
    if (!m || !out || nx < 2 || ny < 2 || (int64_t)nx * ny >= (1LL << 31)) {
        hs_set_error("hs_square_vertex_counts: bad arguments (need m, out and a lattice of at least 2 x 2 cells)");
        return HS_EINVAL;
    }
    return hs_square_vertex_counts_impl(m, nx, ny, out, (cudaStream_t)stream);
}

int hs_progress_disarm(HsCounters *C, void *stream) {
    if (!C) { hs_set_error("hs_progress_disarm: null counters"); return HS_EINVAL; }
    return hs_progress_disarm_impl(C, (cudaStream_t)stream);
}

int hs_region_readout(const int8_t *m, int32_t nx, int32_t ny, int32_t n_regions, const int32_t *rects, const double *wx,
                      const double *wy, const double *norm, double *out, void *stream) {
    if (!m || nx <= 0 || ny <= 0 || n_regions <= 0 || !rects || !wx || !norm || !out) {
        hs_set_error("hs_region_readout: bad arguments");
        return HS_EINVAL;
    }
    return hs_region_readout_impl(m, nx, ny, n_regions, rects, wx, wy, norm, out, (cudaStream_t)stream);
}

int hs_segments_copy(void *staged, const HsSegment *segs, int32_t n, int32_t to_device, void *stream) {
    if (n < 0 || (n > 0 && (!staged || !segs))) { hs_set_error("hs_segments_copy: bad arguments"); return HS_EINVAL; }
    if (n == 0) return HS_OK;
    return hs_segments_copy_impl(staged, segs, n, to_device ? 1 : 0, (cudaStream_t)stream);
}

int hs_engine_run(const HsInstance *insts, int32_t n_inst, int32_t cluster_size, int32_t n_clusters, int32_t *work,
                  void *stream) {
    if (!insts || !work || n_inst < 0 || n_clusters <= 0) { hs_set_error("hs_engine_run: bad arguments"); return HS_EINVAL; }
    if (n_inst == 0) return HS_OK;
    return hs_launch_engine(insts, n_inst, cluster_size, n_clusters, work, HS_ENGINE_WS_DEFAULT, nullptr,
                            (cudaStream_t)stream);
}

int hs_engine_run_ws(const HsInstance *insts, int32_t n_inst, int32_t cluster_size, int32_t n_clusters, int32_t *work,
                     int32_t ws_bytes, int64_t *elapsed_ns, void *stream) {
    if (!insts || !work || n_inst < 0 || n_clusters <= 0) {
        hs_set_error("hs_engine_run_ws: bad arguments");
        return HS_EINVAL;
    }
    if (ws_bytes < 0 || ws_bytes > HS_ENGINE_WS_MAX) {
        hs_set_error("hs_engine_run_ws: workspace of %d bytes outside [0, %d]", (int)ws_bytes, HS_ENGINE_WS_MAX);
        return HS_EINVAL;
    }
    if (n_inst == 0) return HS_OK;
    return hs_launch_engine(insts, n_inst, cluster_size, n_clusters, work, ws_bytes,
                            reinterpret_cast<long long *>(elapsed_ns), (cudaStream_t)stream);
}

int hs_engine_max_clusters(int32_t cluster_size) { return hs_engine_max_clusters_impl(cluster_size); }

int hs_exchange_energy(const HsLattice *L, float *E, float *E_perp, void *stream) {
    int rc = check_lattice(L, "hs_exchange_energy");
    if (rc) return rc;
    if (!L->has_exchange || !E) { hs_set_error("hs_exchange_energy: no exchange energy / output"); return HS_EINVAL; }
    return hs_launch_exchange_energy(*L, E, E_perp, (cudaStream_t)stream);
}

int hs_switch_energy(const HsLattice *L, float *dE, void *stream) {
    int rc = check_lattice(L, "hs_switch_energy");
    if (rc) return rc;
    if (!dE) { hs_set_error("hs_switch_energy: null output"); return HS_EINVAL; }
    return hs_launch_switch_energy(*L, dE, (cudaStream_t)stream);
}

}  // extern "C"
