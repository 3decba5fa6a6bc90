/*
 * hotspice_b200.h — C ABI of the B200 (sm_100a) kinetic Monte Carlo engine.
 *
 * Every entry point is `extern "C"`, takes plain pointers/sizes and an explicit CUDA
 * stream (cudaStream_t passed as void*), returns an int status (HS_OK or a negative code,
 * message via hs_last_error) and never allocates device memory: all buffers, including
 * scratch, belong to the caller (the Python host layer allocates them as torch tensors).
 * Launches are asynchronous; nothing here synchronises the stream.
 *
 * Reference interfaces each entry point replaces (paths inside the Hotspice project):
 *   hs_dipolar_update        DipolarEnergy.update_single / update_multiple
 *                            (hotspice/energies.py:310-329, 331-366)
 *   hs_dipolar_full_direct   DipolarEnergy.update (hotspice/energies.py:290-308), direct sum
 *   hs_dipolar_full_igemm    DipolarEnergy.update as a tensor-core implicit GEMM
 *   hs_neel_step             Magnets._update_Néel + E_barrier + update_energy
 *                            (hotspice/core.py:679-709, 625-656, 241-253)
 *   hs_metropolis_step       Magnets._update_Metropolis + select/_select_grid/_select_single/
 *                            _select_Poisson (hotspice/core.py:659-677, 456-570)
 *   hs_wolff_step            Magnets._update_Wolff + _select_cluster_exchange
 *                            (hotspice/core.py:711-718, 588-602)
 *   hs_minimize_all / hs_relax_check
 *                            Magnets._minimize_all / relax (hotspice/core.py:799-861)
 *   hs_minimize_step         one iteration of Magnets.minimize (hotspice/core.py:763-797)
 *   hs_zeeman_set / hs_progress_arm / hs_region_readout
 *                            the input / output steps of hotspice/io.py:193-500
 *   hs_square_vertex_counts  count_square_vertices (examples/IP_SquareVertices.py:19-35)
 *   hs_exchange_energy       ExchangeEnergy.update (hotspice/energies.py:771-781)
 *   hs_philox_uniform        the variate stream that replaces numpy.random in the hot path
 */
#ifndef HOTSPICE_B200_H
#define HOTSPICE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------------------ */
#define HS_OK          0
#define HS_EINVAL     -1   /* bad argument (size, pointer, unsupported combination)      */
#define HS_ENOMEM     -2   /* caller-provided scratch too small                           */
#define HS_ETIMEDOUT  -3   /* a bounded device loop gave up (flag in HsCounters.status)   */
#define HS_ECUDA      -4   /* CUDA runtime error (launch failure etc.)                     */
#define HS_ERANGE     -5   /* size beyond a compiled-in maximum                           */

/* device-side status bits written to HsCounters.status */
#define HS_ST_SELECT_RETRY   1   /* select() retried too often (no occupied sample)        */
#define HS_ST_SWITCH_OVERFLOW 2  /* more switches than the switch list holds               */
#define HS_ST_POISSON_OVERFLOW 4 /* Poisson-disc grid/queue capacity exceeded              */
#define HS_ST_WOLFF_OVERFLOW 8   /* Wolff frontier capacity exceeded                       */
#define HS_ST_STEP_CAP       16  /* a device-armed progress() run used its whole per-launch step
                                    budget before its stop rule held (set by the next
                                    hs_progress_arm / hs_progress_disarm)                     */

/* Dynamic shared workspace of an engine CTA: hs_engine_run's size, and the largest accepted. */
#define HS_ENGINE_WS_DEFAULT (64 * 1024)
#define HS_ENGINE_WS_MAX (160 * 1024)
/* Per-launch step budget of a progress() run in hs_engine_run when HsInstance.steps is 0. */
#define HS_PROGRESS_STEPS_MAX (1 << 22)

/* update schemes / selection / barrier (SimParams values, hotspice/core.py:29-41) */
#define HS_SCHEME_NEEL        0
#define HS_SCHEME_METROPOLIS  1
#define HS_SCHEME_WOLFF       2
#define HS_SAMPLE_SINGLE      0
#define HS_SAMPLE_GRID        1
#define HS_SAMPLE_POISSON     2
#define HS_BARRIER_SIMPLE     0
#define HS_BARRIER_PARABOLIC  1

/* update semantics of hs_dipolar_update */
#define HS_UPDATE_SINGLE   0   /* add window, then negate E at the switch (update_single)   */
#define HS_UPDATE_MULTIPLE 1   /* negate E at all switches, then add windows (update_multiple) */

/*
 * One lattice instance. All (ny, nx) fields are dense row-major device arrays.
 * Pointers that a configuration does not use are NULL.
 */
typedef struct HsLattice {
    /* -- 8-byte members ---------------------------------------------------------------- */
    int8_t       *m;            /* spins -1/0/+1                                            */
    const int8_t *occ;          /* occupation 0/1                                           */
    float        *mm;           /* m * moment (dipolar source field)                        */
    const float  *moment;       /* magnetic moment [A m^2]                                  */
    const int32_t *nonzero;     /* (n_occ) flat indices of occupied cells, row-major         */
    const int32_t *sub_of;      /* (uy*ux) unit-cell site -> kernel number, or -1           */
    const float  *E_B;          /* anisotropy barrier [J]                                    */
    const float  *beta;         /* 1/(kB T) [1/J]                                            */
    const float  *K;            /* dipolar kernels (n_sub, 2wy+1, 2wx+1), prefactor excluded */
    const float  *Kpo;          /* "perp-other" kernels, same shape, or NULL                 */
    const float  *Kps;          /* "perp-self" kernels (full recompute only), or NULL        */
    double       *E_dip;        /* dipolar energy [J] (FP64 accumulator of FP32 increments)  */
    double       *E_dip_perp;   /* dipolar perpendicular energy, or NULL                     */
    const float  *zee;          /* Zeeman E_factor (E = m * zee), or NULL                    */
    const float  *zee_perp;     /* Zeeman E_factor_perp, or NULL                             */
    const float  *orient;       /* (ny, nx, 2) orientation, in-plane exchange only, or NULL */
    const double *wolff_bond;   /* bond[c] = 1 - exp(-2 J / kBT * c), c = 0..24, uniform T, or NULL */
    double        beta_uniform; /* 1/(kB T) when T is uniform, else 0                        */
    double        J;            /* exchange coupling [J]                                     */
    double        dip_pref;     /* DipolarEnergy.prefactor                                   */
    double        m_perp_factor;
    uint64_t      seed;         /* Philox key                                                */
    /* -- 4-byte members ---------------------------------------------------------------- */
    int32_t nx, ny;
    int32_t ux, uy;             /* unit cell                                                 */
    int32_t pbc;
    int32_t in_plane;
    int32_t use_perp;           /* USE_PERP_ENERGY                                           */
    int32_t n_occ;
    int32_t barrier_method;     /* HS_BARRIER_*                                              */
    int32_t has_dipolar;
    int32_t dip_wx, dip_wy;     /* kernel window half-widths                                 */
    int32_t dip_wrap;           /* 1: PBC with a cropped (minimum-image) window              */
    int32_t n_sub;
    int32_t has_exchange;
    int32_t nn_h, nn_w;         /* exchange nearest-neighbour mask size (odd, <= 5x5)        */
    int32_t trunc_cutoff;       /* SIMULTANEOUS_SWITCHES_CONVOLUTION_OR_SUM_CUTOFF           */
    int32_t trunc_size;         /* REDUCED_KERNEL_SIZE                                       */
    int32_t dip_keep_perp_sign; /* 1: HS_UPDATE_MULTIPLE leaves E_dip_perp of the switched cells
                                   unnegated (DiMonopolarEnergy.update_multiple,
                                   hotspice/energies.py:718-719); 0: negated (DipolarEnergy)   */
    int8_t  nn[28];             /* nearest-neighbour mask, row-major                         */
} HsLattice;

/* Device-resident per-instance counters (one struct in device memory). */
typedef struct HsCounters {
    double   t;            /* simulated time [s]                                            */
    double   t0, mc0;      /* progress(): t and MCsteps at the start                         */
    double   t_max, mc_max;/* progress(): limits (t_max also bounds a single Néel step)      */
    int64_t  switches;
    int64_t  attempted;
    uint64_t rng_call;     /* next Philox call number                                        */
    int32_t  status;       /* HS_ST_* bits                                                    */
    int32_t  done;         /* progress(): stop condition reached                              */
    int32_t  progress;     /* 1: evaluate the progress() stop rule before every step          */
    int32_t  n_sw;         /* switches written by the last step                               */
    int32_t  epoch;        /* Wolff cluster stamp                                             */
    int32_t  steps;        /* steps executed                                                  */
    double   bmin;         /* Néel: global minimum barrier of the last step                   */
    double   last_time;    /* Néel: switching time drawn in the last step                     */
    int64_t  near_threshold; /* decisions whose FP32 margin was below the stated tolerance   */
    double   reserved[4];
} HsCounters;

/* Switch record list written by a step (device memory, capacity `cap`). */
typedef struct HsSwitchList {
    int32_t *y;
    int32_t *x;
    int32_t *mode;         /* 0: exact window, 1: truncated (REDUCED_KERNEL_SIZE) window      */
    int32_t  cap;
    int32_t  pad;
} HsSwitchList;

/* Metropolis selection plan, precomputed on the host from the geometry (hotspice/core.py:506-540). */
typedef struct HsGridPlan {
    const int32_t *phase_off;   /* (ux*uy + 1) offsets into phase_yx per supercell phase         */
    const int32_t *phase_yx;    /* packed (oy << 16 | ox) occupied offsets inside one supercell   */
    int32_t Rx, Ry;             /* supercell size in cells                                       */
    int32_t snx, sny;           /* supercells per axis (every second one is sampled)             */
    int32_t n_sc;               /* sampled supercells                                            */
    int32_t sample_scheme;      /* HS_SAMPLE_*                                                   */
    double  r_cells;            /* Poisson-disc radius in cell units                             */
    int32_t poisson_k;          /* dart throws per active point                                  */
    int32_t metropolis_time;    /* SimParams.METROPOLIS_TIME                                     */
    double  attempt_freq;
} HsGridPlan;

/* One lattice instance of a persistent engine launch (device memory array of these). */
typedef struct HsInstance {
    HsLattice    L;
    HsGridPlan   P;             /* Metropolis selection plan                                  */
    HsSwitchList sw;
    HsCounters  *C;             /* device counters of this instance                           */
    void        *scratch;       /* Metropolis or Wolff working arrays (see *_scratch_bytes)   */
    int64_t      scratch_bytes;
    int64_t      steps;         /* steps to run when C->progress == 0; when C->progress == 1,
                                   the most steps this launch makes (0: HS_PROGRESS_STEPS_MAX) */
    double       attempt_freq;
    int32_t      scheme;        /* HS_SCHEME_*                                                */
    int32_t      flags;         /* HS_INST_* bits                                             */
} HsInstance;

/* HsInstance.flags: run this instance on one CTA of its cluster. In a launch with clusters of
 * more than one CTA, the first flagged instance a cluster claims splits it: from then on each
 * of its CTAs claims and runs instances alone. List flagged instances after all others. */
#define HS_INST_ONE_CTA 1

/* ---- library ------------------------------------------------------------------------- */
int hs_version(void);
int hs_last_error(char *buf, int len);
/* Sizes of the ABI structs, so bindings can check their mirrors; the first n of: sizeof
 * HsLattice, HsCounters, HsSwitchList, HsGridPlan, offsetof(HsLattice, nx), HsInstance,
 * HsSegment. */
int hs_struct_sizes(int32_t *out, int n);

/* n doubles u53 of Philox call `call` into out (device). */
int hs_philox_uniform(uint64_t seed, uint64_t call, int32_t n, double *out, void *stream);

/* ---- (a) incremental dipolar update --------------------------------------------------- */
/* Applies the n switches listed in `sw` (device count *n_sw_dev, or n_host if n_sw_dev is
 * NULL) to E_dip / E_dip_perp. m and mm must already hold the flipped spins. */
int hs_dipolar_update(const HsLattice *L, const HsSwitchList *sw, const int32_t *n_sw_dev,
                      int32_t n_host, int32_t semantics, const HsCounters *C, void *stream);

/* ---- (b) full dipolar recompute ---------------------------------------------------------- */
/* Direct sum over the kernel window. fp64 != 0 accumulates in double, otherwise in float.
 * Writes E64/Ep64 when given, else L->E_dip / L->E_dip_perp. */
int hs_dipolar_full_direct(const HsLattice *L, int32_t fp64, double *E64, double *Ep64, void *stream);
/* Tensor-core implicit GEMM (tcgen05, split-BF16 kernel, FP32 accumulation in TMEM), the
 * counterpart of DipolarEnergy.update (hotspice/energies.py:290-308) for the full, uncropped
 * kernel (dip_wx = nx-1, dip_wy = ny-1, no wrap) and a uniform moment over the occupied cells.
 * nsplit (1..3) BF16 terms of the FP32 kernel. Writes L->E_dip (and E_dip_perp).
 * `scratch` holds the split kernels and BF16 spins (hs_igemm_scratch_bytes); its last 256 bytes
 * start with an int32 status word, valid once the stream has reached the end of the call:
 * 0 = ok, bit 0 = a pipeline wait timed out, bit 1 = the moment is not uniform (E is wrong). */
int64_t hs_igemm_scratch_bytes(const HsLattice *L, int32_t nsplit);
int hs_dipolar_full_igemm(const HsLattice *L, int32_t nsplit, void *scratch, int64_t scratch_bytes, void *stream);

/* Limit, in ns of wall time, of one pipeline wait inside hs_dipolar_full_igemm (0: the default,
 * 4 s). A wait that runs out sets bit 0 of the call's status word and the kernel ends cleanly (its
 * copies land, its MMAs finish, TMEM is freed). No reference counterpart: a safety bound of this
 * library, shortened only to test that path. Applies to later calls of this process. */
int hs_set_wait_limit(uint64_t ns);

/* ---- (c) Néel-Arrhenius step ------------------------------------------------------------- */
int64_t hs_neel_scratch_bytes(const HsLattice *L);
int hs_neel_step(const HsLattice *L, HsCounters *C, const HsSwitchList *sw, double attempt_freq,
                 void *scratch, int64_t scratch_bytes, void *stream);

/* ---- (d) Metropolis step (grid / single / Poisson-disc selection) ------------------------ */
int64_t hs_metropolis_scratch_bytes(const HsLattice *L, const HsGridPlan *P);
int hs_metropolis_step(const HsLattice *L, HsCounters *C, const HsSwitchList *sw, const HsGridPlan *P,
                       void *scratch, int64_t scratch_bytes, void *stream);

/* Allocation-free variant of hs_metropolis_step (no counterpart in the reference). For callers
 * that cannot allocate device memory: the working arrays live in a fixed 4 MiB device array
 * inside the library, one per GPU, kept until the process exits. The first call on a device
 * (with that device current) looks up the array's address; make it before any stream capture.
 * Returns HS_ERANGE when the selection plan needs more than 4 MiB (hs_metropolis_scratch_bytes).
 * All calls share the array: calls that overlap on the GPU race. */
int hs_metropolis_step_noalloc(const HsLattice *L, HsCounters *C, const HsSwitchList *sw, const HsGridPlan *P,
                               void *stream);

/* ---- (e) Wolff cluster step (exchange-only lattices) ------------------------------------- */
int64_t hs_wolff_scratch_bytes(const HsLattice *L);
int hs_wolff_step(const HsLattice *L, HsCounters *C, const HsSwitchList *sw,
                  void *scratch, int64_t scratch_bytes, void *stream);

/* ---- relaxation: relax() / _minimize_all() / minimize() (hotspice/core.py:763-861) ---------- */
/* One scratch layout serves all of these; its first 8 bytes are {int32 done; int32 sweeps}:
 * `done` is set when relax()'s stop rule (or minimize()'s) has fired, after which every call
 * below does nothing until the next hs_relax_begin / hs_minimize_begin; `sweeps` counts the
 * relax sweeps made. Switch list capacity: nx * ny. */
int64_t hs_relax_scratch_bytes(const HsLattice *L);
/* Start relax(): clears the stop state, records m as the state "two sweeps before". */
int hs_relax_begin(const HsLattice *L, void *scratch, int64_t scratch_bytes, void *stream);
/* One _minimize_all sweep (core.py:799-825): draws the subgrid order (one Philox call, a
 * stable argsort of (2ux)(2uy) variates, or of 1 when `simultaneous`), then for each subgrid
 * switches every magnet with switch_energy < 0 (ignore_barrier) or switch_energy / 2 + E_B < 0,
 * and updates the energies (DipolarEnergy.update_single / update_multiple semantics). */
int hs_minimize_all(const HsLattice *L, HsCounters *C, const HsSwitchList *sw, int32_t ignore_barrier,
                    int32_t simultaneous, void *scratch, int64_t scratch_bytes, void *stream);
/* The two halves of hs_minimize_all: the order, then subgrid i (0 <= i < number of subgrids). */
int hs_relax_permute(const HsLattice *L, HsCounters *C, int32_t simultaneous, void *scratch,
                     int64_t scratch_bytes, void *stream);
int hs_relax_subset(const HsLattice *L, HsCounters *C, const HsSwitchList *sw, int32_t i,
                    int32_t ignore_barrier, int32_t simultaneous, void *scratch, int64_t scratch_bytes,
                    void *stream);
/* relax()'s stop rule after a sweep (core.py:842-857): nothing switched, the state equals the
 * one two sweeps before, or n_max = int(sqrt(nx^2 + ny^2)) sweeps were made. */
int hs_relax_check(const HsLattice *L, HsCounters *C, int32_t n_max, void *scratch, int64_t scratch_bytes,
                   void *stream);
/* Start minimize(): clears the stop state and the per-magnet pick counts. */
int hs_minimize_begin(const HsLattice *L, void *scratch, int64_t scratch_bytes, void *stream);
/* One iteration of minimize(ignore_barrier=True) (core.py:771-797): with n magnets whose
 * switch_energy < -kBT, switches ceil(frac n) of them, chosen by one Philox call over n
 * elements (the smallest keys); else switches the first argmin of switch_energy if it is < 0
 * and was not picked three times; else sets `done`. */
int hs_minimize_step(const HsLattice *L, HsCounters *C, const HsSwitchList *sw, double frac, void *scratch,
                     int64_t scratch_bytes, void *stream);

/* ---- reservoir input / output stepping (hotspice/io.py:193-500) ------------------------------ */
/* ZeemanEnergy.set_field (hotspice/energies.py:97-118) in place on the device: with
 * B = magnitude * pattern[i] (pattern NULL: 1) at `angle`, E_factor = -moment (Bx ox + By oy) and
 * E_factor_perp = -moment (By ox - Bx oy) in plane, E_factor = -moment B out of plane. moment and
 * orient (ny, nx, 2) are FP64; E_factor / E_factor_perp (FP64, may be NULL) and zee / zee_perp
 * (the FP32 copies HsLattice points at) are overwritten. */
int hs_zeeman_set(int64_t n_cells, int32_t in_plane, const double *moment, const double *orient, const float *pattern,
                  double magnitude, double angle, double *E_factor, double *E_factor_perp, float *zee, float *zee_perp,
                  void *stream);
/* Arms progress(t_max, MCsteps_max) (hotspice/core.py:736-760) from the device counters
 * (t0 = t, mc0 = attempted / n_occ); a following hs_engine_run advances until the stop rule.
 * At least one limit must be finite. If a previous armed run is still unfinished (it used its
 * step budget), HS_ST_STEP_CAP is set in C->status first. */
int hs_progress_arm(HsCounters *C, int32_t n_occ, double t_max, double MCsteps_max, void *stream);
/* Ends a device-armed progress(): progress = 0, done = 0 (plain steps run again); sets
 * HS_ST_STEP_CAP when the armed run had not finished. */
int hs_progress_disarm(HsCounters *C, void *stream);
/* Coarse-grained readout (RegionalOutputReader / OOPSquareChessOutputReader.read_state,
 * hotspice/io.py:362-380, 438-446): for region r with cell rectangle rects[4r..4r+3] =
 * {y0, y1, x0, x1} (half-open, clipped to the lattice), out[r] = sum m * wx / norm[r] and, when
 * wy is not NULL, out[n_regions + r] = sum m * wy / norm[r]. */
int hs_region_readout(const int8_t *m, int32_t nx, int32_t ny, int32_t n_regions, const int32_t *rects, const double *wx,
                      const double *wy, const double *norm, double *out, void *stream);

/* Vertex-type counts of an in-plane square ASI state (count_square_vertices,
 * examples/IP_SquareVertices.py:19-35): vertices are the cells with even x and y, each with its
 * four neighbouring magnets (periodic wrap); out[0..3] (device int64, overwritten) = the numbers
 * of type 1 (flower), 2, 3 and 4 vertices. */
int hs_square_vertex_counts(const int8_t *m, int32_t nx, int32_t ny, int64_t *out, void *stream);

/* ---- packed state transfer for batches (no reference counterpart: it replaces the per-array
 * host<->device copies of a batch's start states and results) ---------------------------------- */
/* One segment: `bytes` bytes at offset `staged` of a staging buffer <-> device address `device`.
 * Segments of at most HS_SEGMENT_MAX bytes spread the copy over the SMs (one CTA per segment). */
#define HS_SEGMENT_MAX 65536
typedef struct HsSegment {
    int64_t  staged;
    uint64_t device;
    int64_t  bytes;
} HsSegment;
/* Scatters the device-resident staging buffer `staged` into the segments' addresses
 * (to_device = 1) or gathers them into it (to_device = 0); `segs` is a device array of n
 * segments. With one host<->device copy of the staging buffer this moves a whole batch's state
 * in two operations. */
int hs_segments_copy(void *staged, const HsSegment *segs, int32_t n, int32_t to_device, void *stream);

/* ---- persistent multi-instance engine -------------------------------------------------------- */
/* Advances n_inst instances (device array `insts`) in one launch of n_clusters thread-block
 * clusters of `cluster_size` CTAs (1, 2, 4, 8 or 16). Each cluster claims instances from the
 * device counter `work` (reset by this call) and runs each instance's step budget, or, when
 * C->progress is set, until its progress() stop rule holds (C->done = 1), a step reports a
 * status bit, or the launch's step budget (HsInstance.steps, else HS_PROGRESS_STEPS_MAX) is
 * used up; then C->done stays 0 and a further launch continues the run. Every launch ends.
 * Replaces repeated update() calls (hotspice/core.py:604-622, 736-760) for many simulations at
 * once. */
int hs_engine_run(const HsInstance *insts, int32_t n_inst, int32_t cluster_size, int32_t n_clusters,
                  int32_t *work, void *stream);
/* hs_engine_run with an explicit dynamic shared workspace of ws_bytes per CTA (0 to
 * HS_ENGINE_WS_MAX; hs_engine_run uses HS_ENGINE_WS_DEFAULT). A Poisson-disc Metropolis
 * instance keeps its sampler arrays (24 * background-grid cells + 64 bytes) there when they
 * fit, else in its scratch; the workspace takes L1 capacity from every other phase, so a
 * launch without Poisson-disc instances passes 0. Results do not depend on ws_bytes.
 * elapsed_ns (device memory, n_inst entries, or NULL): per instance of `insts`, the device
 * wall time (ns) its cluster spent on it in this launch, from claim to counter write-back. */
int hs_engine_run_ws(const HsInstance *insts, int32_t n_inst, int32_t cluster_size, int32_t n_clusters,
                     int32_t *work, int32_t ws_bytes, int64_t *elapsed_ns, void *stream);
/* Number of clusters of `cluster_size` CTAs that can be resident at once (occupancy query). */
int hs_engine_max_clusters(int32_t cluster_size);

/* ---- helpers ------------------------------------------------------------------------------- */
/* Exchange energy field E (and E_perp when use_perp) from the current spins. */
int hs_exchange_energy(const HsLattice *L, float *E, float *E_perp, void *stream);
/* Total switch energy dE = -2 E_total at every cell (NaN where unoccupied), for the API. */
int hs_switch_energy(const HsLattice *L, float *dE, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* HOTSPICE_B200_H */
