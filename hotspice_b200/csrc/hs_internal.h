// Internal host-side declarations shared by the .cu translation units.
#pragma once

#include <cuda_runtime.h>
#include <algorithm>
#include <stdint.h>

#include "../../include/hotspice_b200.h"

// error reporting (hs_capi.cu)
void hs_set_error(const char *fmt, ...);
int hs_check_launch(const char *what);

// launchers
int hs_launch_dipolar_update(const HsLattice &L, const HsSwitchList &sw, const int32_t *n_sw_dev, int n_host,
                             int semantics, const HsCounters *C, cudaStream_t st);
int hs_launch_dipolar_full_direct(const HsLattice &L, int fp64, double *E64, double *Ep64, cudaStream_t st);
int64_t hs_neel_scratch(const HsLattice &L);
int hs_launch_neel(const HsLattice &L, HsCounters *C, const HsSwitchList &sw, double attempt_freq,
                   void *scratch, int64_t scratch_bytes, cudaStream_t st);
int64_t hs_metropolis_scratch(const HsLattice &L, const HsGridPlan &P);
// Validation shared by every Metropolis entry point (hs_capi.cu): the lattice, the plan and,
// for Poisson-disc plans, a finite radius and a background grid of at most HS_POISSON_GRID_MAX
// cells; the second form also checks the counters and the switch list.
int hs_check_metropolis_plan(const HsLattice *L, const HsGridPlan *P, const char *who);
int hs_check_metropolis_args(const HsLattice *L, const HsCounters *C, const HsSwitchList *sw, const HsGridPlan *P,
                             const char *who);
int hs_launch_metropolis(const HsLattice &L, HsCounters *C, const HsSwitchList &sw, const HsGridPlan &P,
                         void *scratch, int64_t scratch_bytes, cudaStream_t st);
int64_t hs_wolff_scratch(const HsLattice &L);
int hs_launch_wolff(const HsLattice &L, HsCounters *C, const HsSwitchList &sw, void *scratch,
                    int64_t scratch_bytes, cudaStream_t st);
int hs_launch_exchange_energy(const HsLattice &L, float *E, float *Ep, cudaStream_t st);
int hs_launch_switch_energy(const HsLattice &L, float *dE, cudaStream_t st);
int hs_launch_philox(uint64_t seed, uint64_t call, int32_t n, double *out, cudaStream_t st);
int64_t hs_igemm_scratch(const HsLattice &L, int nsplit);
int hs_launch_igemm(const HsLattice &L, int nsplit, void *scratch, int64_t scratch_bytes, cudaStream_t st);
int hs_set_wait_limit_impl(unsigned long long ns);

int64_t hs_relax_scratch(const HsLattice &L);
int hs_relax_begin_impl(const HsLattice &L, void *scratch, int64_t bytes, cudaStream_t st);
int hs_relax_permute_impl(const HsLattice &L, HsCounters *C, int simultaneous, void *scratch, int64_t bytes,
                          cudaStream_t st);
int hs_relax_subset_impl(const HsLattice &L, HsCounters *C, const HsSwitchList &sw, int i, int ignore_barrier,
                         int simultaneous, void *scratch, int64_t bytes, cudaStream_t st);
int hs_relax_check_impl(const HsLattice &L, HsCounters *C, int n_max, void *scratch, int64_t bytes, cudaStream_t st);
int hs_minimize_begin_impl(const HsLattice &L, void *scratch, int64_t bytes, cudaStream_t st);
int hs_minimize_step_impl(const HsLattice &L, HsCounters *C, const HsSwitchList &sw, double frac, void *scratch,
                          int64_t bytes, cudaStream_t st);

int hs_zeeman_set_impl(int64_t n_cells, int in_plane, const double *moment, const double *orient, const float *pattern,
                       double magnitude, double angle, double *ef, double *efp, float *ef32, float *efp32, cudaStream_t st);
int hs_progress_arm_impl(HsCounters *C, int n_occ, double t_max, double mc_max, cudaStream_t st);
int hs_progress_disarm_impl(HsCounters *C, cudaStream_t st);
int hs_region_readout_impl(const int8_t *m, int nx, int ny, int R, const int32_t *rects, const double *wx,
                           const double *wy, const double *norm, double *out, cudaStream_t st);

int hs_square_vertex_counts_impl(const int8_t *m, int nx, int ny, int64_t *out, cudaStream_t st);

int hs_segments_copy_impl(void *staged, const HsSegment *segs, int n, int to_device, cudaStream_t st);

int hs_launch_engine(const HsInstance *insts, int n_inst, int cluster_size, int n_clusters, int *work, int ws_bytes,
                     long long *elapsed_ns, cudaStream_t st);
int hs_engine_max_clusters_impl(int cluster_size);

inline int64_t hs_align_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }
