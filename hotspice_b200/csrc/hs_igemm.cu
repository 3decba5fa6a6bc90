// (b) Full dipolar recompute as an implicit GEMM on the sm_100a tensor cores (tcgen05).
//
//   out_s[y, x] = sum_{y', x'} K_s[y' - y, x' - x] m[y', x']         (hotspice/energies.py:290-308)
//   E[y, x]     = pref * mu^2 * m[y, x] * out_{s(y,x)}[y, x]          (uniform moment mu)
//
// For one output tile (128 columns x0.., 256 rows y0..) and one kernel-row offset dy, the
// sum over x' is a GEMM D[M=128, N=256] += A[128, K] * B[K, 256] with
//   B[k, n] = m[y0 + n + dy, x'_k]                     (spins, exact in BF16)
//   A[m', k] = K_s[dy, x'_k - x(m') + nx - 1],  x(m') = x0 + 127 - m'   (rows reversed)
// Reversing the rows turns the Toeplitz operand into a Hankel one: its 8x8 core matrices
// depend only on (i + j) (i = 8-row group, j = 8-column group), so one contiguous "strip" of
// core matrices per kernel row, addressed with LBO = SBO = 128 bytes in a no-swizzle K-major
// shared-memory descriptor, serves every (x0, K-block) combination: the A operand of a stage
// is a 23-core-matrix (2944-byte) slice of that strip, copied with one bulk copy.
// The B operands of consecutive dy are the same spin rows shifted by one row. The spins are
// stored column-group-major (8 columns x all rows, 16 bytes per row), so a "band" of 512 rows
// of one 64-column K-block sits in shared memory as 8 columns of 16-byte rows, and the B
// operand of any dy within the band's 256 offsets is a no-swizzle K-major descriptor that
// starts 16 * (dy - band start) bytes in (SBO = 128 B along N, LBO = 8 KB along K): one
// 64 KB band load serves up to 256 stages.
// The FP32 kernel is split into nsplit BF16 terms (hi + mid [+ lo]); the near offsets (within
// NEAR_W cells, periodically when PBC) are left out of the strips and summed in FP64 by the
// finalize, so the FP32 tensor-memory accumulator only carries the far field. Every CHUNK
// stages the accumulator is flushed into FP64 partial sums (two TMEM accumulators alternate,
// so the MMAs continue while the epilogue drains); the stages of a tile are split over KS
// CTAs, each with its own partial-sum slot, summed in a fixed order by the finalize
// (deterministic).
//
// Warp roles (256 threads): warp 0 producer (bulk copies), warp 1 MMA issuer and TMEM owner,
// warps 4-7 epilogue (TMEM lanes 0-127). Every mbarrier wait is bounded in time (a pipeline
// wait by hs_set_wait_limit, 4 s by default); on a timeout the kernel records ST_TIMEOUT in its
// status word, lets its copies land and its MMAs finish (those waits keep the 4 s bound) and
// frees TMEM.
#include <cuda_bf16.h>

#include "hs_common.cuh"
#include "hs_internal.h"

namespace {

constexpr int BM = 128, BN = 256, BK = 64, STAGES = 6, NT = 256;
constexpr int CORE_PER_STAGE = 23;                  // (BM/8 - 1) + (BK/8 - 1) + 1
constexpr int A_BYTES = CORE_PER_STAGE * 128;       // 2944
constexpr int A_SLOT = 3072;                        // per split
constexpr int MAX_SPLIT = 3;
constexpr int STAGE_BYTES = MAX_SPLIT * A_SLOT;
constexpr int DB = 256;                             // kernel-row offsets per spin band
constexpr int BAND_ROWS = BN + DB;                  // 512
constexpr int KGROUP_BYTES = BAND_ROWS * 16;        // one 8-column group of a band: 8 KB
constexpr int BAND_BYTES = 8 * KGROUP_BYTES;        // 64 KB
constexpr int PAD_LO = 256, PAD_HI = 512;           // zero spin rows below / above the lattice
#ifndef HS_IGEMM_CHUNK
#define HS_IGEMM_CHUNK 64
#endif
constexpr int CHUNK = HS_IGEMM_CHUNK;               // stages per FP32 accumulator chunk
constexpr int SMEM_BYTES = 2 * BAND_BYTES + STAGES * STAGE_BYTES + 1024 + 256;
constexpr uint32_t TMEM_COLS = 512;                 // two 256-column FP32 accumulators
constexpr unsigned long long WAIT_NS = 4000000000ULL;  // a wait gives up after 4 s of wall time
constexpr int NEAR_W = 3;          // offsets within this (periodic) distance in both axes are summed in FP64
constexpr int ST_TIMEOUT = 1;      // a pipeline wait gave up
constexpr int ST_MOMENT = 2;       // the moment is not uniform over the occupied cells

struct IgemmParams {
    const __nv_bfloat16 *strips;   // [U][nsplit][2ny-1][qspan][64]
    const __nv_bfloat16 *spins;    // [P/8][PAD_LO + ny + PAD_HI][8]
    int qspan, qmin, nsplit, sub, P, C, nx, ny, rows;
    int XT, KS, G;                 // column tiles, K-splits per tile, stages per accumulator chunk
    double *acc;                   // [KS][ny][P] FP64 partial sums (one slot per K-split)
    int *status;
    unsigned long long wait_ns;    // limit of a pipeline wait (the drain after an abort keeps WAIT_NS)
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ unsigned long long globaltimer_ns() { return hs_globaltimer_ns(); }

// Parity wait bounded in wall time; returns false when it gave up or another thread aborted.
// `backoff` makes an idle waiter sleep between polls so that it does not steal issue slots.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, volatile int *abort_flag,
                                          unsigned long long limit_ns = WAIT_NS, bool backoff = false) {
    const uint32_t a = smem_u32(bar);
    const unsigned long long t0 = globaltimer_ns();
    for (unsigned it = 0;; ++it) {
        uint32_t ok;
        asm volatile("{\n\t.reg .pred P;\n\tmbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\tselp.u32 %0, 1, 0, P;\n\t}"
                     : "=r"(ok) : "r"(a), "r"(parity) : "memory");
        if (ok) return true;
        if (backoff) __nanosleep(500);
        // the clock is read every 256 polls, or on every poll when the limit was shortened
        if ((it & 255) == 255 || limit_ns < WAIT_NS) {
            if (*abort_flag) return false;
            if (globaltimer_ns() - t0 > limit_ns) { *abort_flag = 1; return false; }
        }
    }
}

__device__ __forceinline__ void bulk_copy(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ uint64_t desc_a_hankel(uint32_t saddr) {
    // K-major, no swizzle; LBO = SBO = 128 B (core matrices indexed by i + j); sm100 version 1
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFF) >> 4);
    d |= (uint64_t)(128 >> 4) << 16;
    d |= (uint64_t)(128 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    return d;  // layout type 0 = SWIZZLE_NONE
}
__device__ __forceinline__ uint64_t desc_b_band(uint32_t saddr) {
    // K-major, no swizzle: 8-row groups 128 B apart (N, SBO), 8-column groups KGROUP_BYTES apart (K, LBO)
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFF) >> 4);
    d |= (uint64_t)(KGROUP_BYTES >> 4) << 16;
    d |= (uint64_t)(128 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}
// kind::f16 instruction descriptor: D = F32, A = B = BF16, both K-major, N = 256, M = 128
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                 ::"r"(tmem), "l"(a), "l"(b), "r"(IDESC), "r"(accumulate));
}
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Stage range of one CTA: tile (xt, yt), K-split ks of the tile's chunks of G stages.
struct Work {
    int x0, y0, dlo, dhi, T, ks, c_begin, n_chunks;
};
__device__ __forceinline__ Work work_of(const IgemmParams &p) {
    Work w;
    const int tile = blockIdx.x / p.KS;
    w.ks = blockIdx.x % p.KS;
    w.x0 = (tile % p.XT) * BM;
    w.y0 = (tile / p.XT) * BN;
    w.dlo = max(-(p.ny - 1), -(w.y0 + BN - 1));
    w.dhi = p.ny - 1 - w.y0;
    w.T = (w.dhi - w.dlo + 1) * p.C;
    const int nch = (w.T + p.G - 1) / p.G, cpk = (nch + p.KS - 1) / p.KS;
    w.c_begin = w.ks * cpk;
    w.n_chunks = max(0, min(nch, w.c_begin + cpk) - w.c_begin);
    return w;
}

// k-th index of [0, n) in the order farthest-from-`near` first (ties: the larger index first).
__device__ __forceinline__ int far_first_index(int k, int n, int near) {
    const int kk = n - 1 - k;                 // position in the nearest-first order
    const int R = n - 1 - near, Lf = near, mm = min(R, Lf);
    if (kk == 0) return near;
    if (kk <= 2 * mm) { const int d = (kk + 1) / 2; return (kk & 1) ? near + d : near - d; }
    const int d = mm + (kk - 2 * mm);
    return R > Lf ? near + d : near - d;
}
// k-th value of [lo, hi] in the order of decreasing |value| (ties: the positive value first).
__device__ __forceinline__ int far_first_value(int k, int lo, int hi) {
    if (lo >= 0) return hi - k;
    if (hi <= 0) return lo + k;
    const int A = hi, B = -lo, D = max(A, B), m = min(A, B);
    if (k < D - m) return A > B ? D - k : -(D - k);
    const int u = k - (D - m);
    if (u < 2 * m) { const int d = m - u / 2; return (u & 1) ? -d : d; }
    return 0;
}

// Stage order of a tile: bands of DB kernel rows (band b covers dy in [dlo + b DB, ...], the
// last one shorter), each swept over the C K-blocks, each (band, K-block) over its rows; bands,
// K-blocks and rows are each visited farthest first, so the largest far-field terms of the
// tile are the last ones added to its FP32 accumulator chunk. Any order of the rows within a
// band reuses the band's spins. `band` numbers the (band, K-block) pairs in visiting order.
struct Stage {
    int dy, cc, off, band, row0;   // off = dy - first row of the band; row0 = first spin row of the band
};
struct StageIter {
    Stage s;
    int p, ci, o;                  // positions: band, K-block, row within the band
    int nb_total, zb, cnear, C, dlo, dhi, y0, lo_b, hi_b, Lb;
    __device__ __forceinline__ void set_band() {
        const int bi = far_first_index(p, nb_total, zb);
        lo_b = dlo + bi * DB;
        hi_b = min(dhi, lo_b + DB - 1);
        Lb = hi_b - lo_b + 1;
    }
    __device__ __forceinline__ void fill() {
        s.dy = far_first_value(o, lo_b, hi_b);
        s.off = s.dy - lo_b;
        s.cc = far_first_index(ci, C, cnear);
        s.band = p * C + ci;
        s.row0 = y0 + lo_b;
    }
    __device__ __forceinline__ StageIter(int t, const Work &w, int C_) {
        C = C_; dlo = w.dlo; dhi = w.dhi; y0 = w.y0;
        const int n_dy = dhi - dlo + 1;
        nb_total = (n_dy + DB - 1) / DB;
        zb = (0 - dlo) / DB;                   // band holding dy = 0
        cnear = min(w.x0 / BK + 1, C - 1);     // K-block holding the tile's centre column
        int acc = 0;
        for (p = 0; p < nb_total; ++p) {
            set_band();
            if (t < acc + Lb * C) break;
            acc += Lb * C;
        }
        if (p == nb_total) { p = nb_total - 1; set_band(); }
        const int r = t - acc;
        ci = r / Lb;
        o = r - ci * Lb;
        fill();
    }
    __device__ __forceinline__ void next() {
        if (++o == Lb) {
            o = 0;
            if (++ci == C) {
                ci = 0;
                if (++p < nb_total) set_band();
            }
        }
        fill();
    }
};

__global__ void __launch_bounds__(NT, 1) igemm_kernel(IgemmParams p) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char *smem = reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
    unsigned char *bands = smem;                          // [2][BAND_BYTES]
    unsigned char *astage = smem + 2 * BAND_BYTES;        // [STAGES][STAGE_BYTES]
    uint64_t *full = reinterpret_cast<uint64_t *>(astage + STAGES * STAGE_BYTES);
    uint64_t *empty = full + STAGES;
    uint64_t *bfull = empty + STAGES;  // [2] band loaded
    uint64_t *bempty = bfull + 2;      // [2] band no longer read by MMAs
    uint64_t *accf = bempty + 2;       // [2] accumulator b complete (MMA -> epilogue)
    uint64_t *acce = accf + 2;         // [2] accumulator b drained (epilogue -> MMA)
    uint64_t *done = acce + 2;         // every issued MMA has completed
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(done + 1);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const Work w = work_of(p);
    const int t_begin = w.c_begin * p.G, t_end = min(w.T, (w.c_begin + w.n_chunks) * p.G);

    if (threadIdx.x == 0) {
        for (int s = 0; s < STAGES; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&accf[b], 1); mbar_init(&acce[b], 128);
            mbar_init(&bfull[b], 1); mbar_init(&bempty[b], 1);
        }
        mbar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)), "r"(TMEM_COLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tmem_slot;
    const size_t row_elems = (size_t)p.qspan * 64;

    if (warp == 0 && lane == 0) {
        // ---------------- producer ----------------
        int issued = 0, nb = -1, prev_band = -1;
        StageIter it(t_begin, w, p.C);
        for (int t = t_begin; t < t_end; ++t, it.next()) {
            const Stage &S = it.s;
            if (S.band != prev_band) {  // next spin band into slot nb & 1
                prev_band = S.band;
                ++nb;
                const int slot = nb & 1;
                if (nb >= 2 && !mbar_wait(&bempty[slot], ((nb >> 1) - 1) & 1, abort_flag, p.wait_ns)) { --nb; break; }
                mbar_expect_tx(&bfull[slot], BAND_BYTES);
                const __nv_bfloat16 *src = p.spins + ((size_t)(S.cc * 8) * p.rows + (S.row0 + PAD_LO)) * 8;
                for (int j = 0; j < 8; ++j)
                    bulk_copy(bands + slot * BAND_BYTES + j * KGROUP_BYTES, src + (size_t)j * p.rows * 8, KGROUP_BYTES, &bfull[slot]);
            }
            const int u = t - t_begin, st = u % STAGES;
            if (u >= STAGES && !mbar_wait(&empty[st], ((u / STAGES) - 1) & 1, abort_flag, p.wait_ns)) break;
            unsigned char *sa = astage + st * STAGE_BYTES;
            mbar_expect_tx(&full[st], p.nsplit * A_BYTES);
            const int q0 = 8 * S.cc - w.x0 / 8 - p.qmin;
            for (int sp = 0; sp < p.nsplit; ++sp) {
                const __nv_bfloat16 *src = p.strips + (((size_t)(p.sub * p.nsplit + sp) * (2 * p.ny - 1) + (S.dy + p.ny - 1)) * row_elems) +
                                           (size_t)q0 * 64;
                bulk_copy(sa + sp * A_SLOT, src, A_BYTES, &full[st]);
            }
            issued = u + 1;
        }
        if (*abort_flag) {  // let the copies still in flight land before the CTA exits (bounded)
            volatile int never = 0;
            for (int u = max(0, issued - STAGES); u < issued; ++u) mbar_wait(&full[u % STAGES], (u / STAGES) & 1, &never);
            for (int n = max(0, nb - 1); n <= nb; ++n) mbar_wait(&bfull[n & 1], (n >> 1) & 1, &never);
        }
    } else if (warp == 1 && lane == 0) {
        // ---------------- MMA issuer: chunk lc accumulates into TMEM columns (lc & 1) * 256 ----------------
        bool ok = true;
        int nb = -1, prev_band = -1;
        StageIter it(t_begin, w, p.C);
        for (int lc = 0; lc < w.n_chunks && ok; ++lc) {
            const int b = lc & 1;
            if (lc >= 2 && !mbar_wait(&acce[b], ((lc >> 1) - 1) & 1, abort_flag, p.wait_ns)) break;
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t d = tmem + (uint32_t)(b * BN);
            const int tb = t_begin + lc * p.G, te = min(t_end, tb + p.G);
            for (int t = tb; t < te; ++t, it.next()) {
                const Stage &S = it.s;
                if (S.band != prev_band) {
                    if (nb >= 0) mma_commit(&bempty[nb & 1]);  // the previous band is free once its MMAs finish
                    prev_band = S.band;
                    ++nb;
                    if (!mbar_wait(&bfull[nb & 1], (nb >> 1) & 1, abort_flag, p.wait_ns)) { ok = false; break; }
                    asm volatile("tcgen05.fence::after_thread_sync;");
                }
                const int u = t - t_begin, st = u % STAGES;
                if (!mbar_wait(&full[st], (u / STAGES) & 1, abort_flag, p.wait_ns)) { ok = false; break; }
                asm volatile("tcgen05.fence::after_thread_sync;");
                const uint32_t sa = smem_u32(astage + st * STAGE_BYTES);
                const uint32_t sb = smem_u32(bands + (nb & 1) * BAND_BYTES) + (uint32_t)(S.off * 16);
                for (int sp = p.nsplit - 1; sp >= 0; --sp)  // smallest split terms first
#pragma unroll
                    for (int ks = 0; ks < BK / 16; ++ks) {
                        const uint64_t a = desc_a_hankel(sa + sp * A_SLOT + ks * 2 * 128);
                        const uint64_t bd = desc_b_band(sb + ks * 2 * KGROUP_BYTES);
                        mma_bf16(d, a, bd, (t != tb || sp != p.nsplit - 1 || ks != 0) ? 1u : 0u);
                    }
                mma_commit(&empty[st]);
            }
            if (ok) mma_commit(&accf[b]);
        }
        mma_commit(done);  // arrives once every MMA issued above has completed
        volatile int never = 0;
        mbar_wait(done, 0, &never);
    } else if (warp >= 4) {
        // ---------------- epilogue: TMEM chunk -> FP64 partial sums of this K-split ----------------
        const int mrow = 32 * (warp - 4) + lane;
        const int x = w.x0 + BM - 1 - mrow;
        double *slot = p.acc + (size_t)w.ks * p.ny * p.P;
        if (w.n_chunks == 0 && x < p.nx) {
            for (int j = 0; j < BN && w.y0 + j < p.ny; ++j) slot[(size_t)(w.y0 + j) * p.P + x] = 0.0;
        }
        for (int lc = 0; lc < w.n_chunks; ++lc) {
            const int b = lc & 1;
            if (!mbar_wait(&accf[b], (lc >> 1) & 1, abort_flag, p.wait_ns, true)) break;
            asm volatile("tcgen05.fence::after_thread_sync;");
            for (int n0 = 0; n0 < BN; n0 += 32) {
                uint32_t v[32];
                const uint32_t addr = tmem + ((uint32_t)(32 * (warp - 4)) << 16) + (uint32_t)(b * BN + n0);
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                             "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                             : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                               "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
                               "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
                               "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                             : "r"(addr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (x < p.nx) {
                    const int jn = min(32, p.ny - (w.y0 + n0));
                    double *col = slot + (size_t)(w.y0 + n0) * p.P + x;
                    if (lc == 0) {
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            if (j < jn) col[(size_t)j * p.P] = (double)__uint_as_float(v[j]);
                    } else {
                        double old[32];
#pragma unroll
                        for (int j = 0; j < 32; ++j) old[j] = j < jn ? col[(size_t)j * p.P] : 0.0;
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            if (j < jn) col[(size_t)j * p.P] = old[j] + (double)__uint_as_float(v[j]);
                    }
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;");
            mbar_arrive(&acce[b]);
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (threadIdx.x == 0 && *abort_flag) atomicOr(p.status, ST_TIMEOUT);
    if (warp == 1) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
    }
}

// E of the cells of sublattice `sub`: pref * mu_i * mu * m_i * (sum of the K-split partials, in
// order, plus the near offsets excluded from the strips, summed here in FP64).
__global__ void igemm_finalize_kernel(const double *acc, int KS, int P, int nx, int ny, int ux, int uy, const int32_t *sub_of,
                                      int sub, const int8_t *m, const float *moment, const unsigned long long *first,
                                      const float *K, int pbc, int w, double pref, double *out) {
    const unsigned long long f = *first;
    const double mu = f == ~0ULL ? 0.0 : (double)moment[f];
    const int64_t n = (int64_t)nx * ny, plane = (int64_t)ny * P;
    const int64_t W = 2 * nx - 1, H = 2 * ny - 1;
    const float *Ks = K + (int64_t)sub * H * W;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int y = (int)(i / nx), x = (int)(i % nx);
        if (sub_of[(y % uy) * ux + (x % ux)] != sub) continue;
        double s = 0.0;
        for (int k = 0; k < KS; ++k) s += acc[k * plane + (int64_t)y * P + x];
        double near = 0.0;
        for (int ddy = -w; ddy <= w; ++ddy) {
            int yy = y + ddy;
            if (pbc) yy = (yy % ny + ny) % ny;
            else if (yy < 0 || yy >= ny) continue;
            for (int ddx = -w; ddx <= w; ++ddx) {
                int xx = x + ddx;
                if (pbc) xx = (xx % nx + nx) % nx;
                else if (xx < 0 || xx >= nx) continue;
                const int mj = m[(int64_t)yy * nx + xx];
                if (mj) near += (double)Ks[(int64_t)(yy - y + ny - 1) * W + (xx - x + nx - 1)] * (double)mj;
            }
        }
        out[i] = pref * (double)moment[i] * mu * (double)m[i] * (s + near);
    }
}

// Is kernel offset d (of a lattice n cells long) within distance w, periodically when pbc?
__device__ __forceinline__ bool near_offset(int64_t d, int n, int pbc, int w) {
    const int64_t a = d < 0 ? -d : d;
    return a <= w || (pbc && n - a <= w);
}

// Split-BF16 Hankel strips: core matrix q of kernel row dy holds K[dy, 8q + (nx - 128) + r + t]
// at element r * 8 + t (zero outside the row, and zero for the near offsets that the finalize
// sums in FP64, so that the FP32 tensor-core accumulator only carries the far field).
__global__ void strips_kernel(const float *K, int nx, int ny, int U, int nsplit, int qspan, int qmin, int pbc, int w,
                              __nv_bfloat16 *out) {
    // one block per kernel row (sublattice s, row dyi); 32-bit index arithmetic within the row
    const int H = 2 * ny - 1, W = 2 * nx - 1;
    const int row = blockIdx.x, s = row / H, dyi = row - s * H;
    const bool near_y = near_offset(dyi - (ny - 1), ny, pbc, w);
    const float *Krow = K + (int64_t)row * W;
    const int n = qspan * 64;
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
        const int rt = e & 63, q = e >> 6;
        const int col = 8 * (q + qmin) + (nx - 128) + (rt >> 3) + (rt & 7);
        float v = (col >= 0 && col < W) ? __ldg(Krow + col) : 0.f;
        if (near_y && near_offset(col - (nx - 1), nx, pbc, w)) v = 0.f;
        float rem = v;
        for (int sp = 0; sp < nsplit; ++sp) {
            const __nv_bfloat16 b = __float2bfloat16_rn(rem);
            rem -= __bfloat162float(b);
            out[(((int64_t)(s * nsplit + sp) * H + dyi) * qspan) * 64 + e] = b;
        }
    }
}

// Index of the first cell holding a spin (its moment is the uniform source moment).
__global__ void first_spin_kernel(const int8_t *m, int64_t n, unsigned long long *first) {
    unsigned long long best = ~0ULL;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (m[i] != 0) { best = (unsigned long long)i; break; }
    for (int o = 16; o; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
    if ((threadIdx.x & 31) == 0 && best != ~0ULL) atomicMin(first, best);
}

// BF16 spins, column-group-major: out[g][PAD_LO + y][e] = m[y][8g + e] (zero outside the
// lattice); flags a non-uniform moment in `status`.
__global__ void spins_bf16_kernel(const int8_t *m, const float *moment, int nx, int ny, int P, int rows,
                                  const unsigned long long *first, __nv_bfloat16 *out, int *status) {
    const int64_t total = (int64_t)(P / 8) * rows * 8;
    const unsigned long long f = *first;
    const float mu0 = f == ~0ULL ? 0.f : moment[f];
    bool bad = false;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int el = (int)(e & 7);
        const int64_t r = (e >> 3) % rows;
        const int g = (int)((e >> 3) / rows);
        const int64_t y = r - PAD_LO;
        const int x = 8 * g + el;
        int mi = 0;
        if (y >= 0 && y < ny && x < nx) {
            mi = m[y * nx + x];
            bad |= (mi != 0 && moment[y * nx + x] != mu0);
        }
        out[e] = __float2bfloat16_rn((float)mi);
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(status, ST_MOMENT);
}

struct Layout {
    int P, C, qspan, qmin, XT, YT, KS, G, rows;
    int64_t strips_bytes, spins_off, spins_bytes, acc_off, acc_bytes, status_off, total;
};

int sm_count() {
    int dev = 0, n = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
}

Layout layout_of(const HsLattice &L, int nsplit) {
    Layout o;
    o.P = (int)hs_align_up(L.nx, BM);
    o.C = o.P / BK;
    o.qspan = o.P / 4 + CORE_PER_STAGE;
    o.qmin = 16 - o.P / 8;
    o.XT = o.P / BM;
    o.YT = (L.ny + BN - 1) / BN;
    o.G = CHUNK;
    o.rows = PAD_LO + L.ny + PAD_HI;
    // K-splits per tile: the most even fill of the SMs (every split keeps at least one chunk,
    // the partial sums stay under 4 GiB)
    const int tiles = o.XT * o.YT, sms = sm_count();
    const int T_min = (L.ny - 1 - (o.YT - 1) * BN - max(-(L.ny - 1), -((o.YT - 1) * BN + BN - 1)) + 1) * o.C;
    const int nch_min = (T_min + o.G - 1) / o.G;
    double best = -1.0;
    o.KS = 1;
    for (int ks = 1; ks <= 16 && ks <= nch_min; ++ks) {
        if ((double)ks * L.ny * o.P * 8 > 4.0e9) break;
        const int64_t ctas = (int64_t)tiles * ks, waves = (ctas + sms - 1) / sms;
        const double eff = (double)ctas / (double)(waves * sms);
        if (eff > best + 1e-9) { best = eff; o.KS = ks; }
    }
    o.strips_bytes = (int64_t)L.n_sub * nsplit * (2 * L.ny - 1) * o.qspan * 128;
    o.spins_off = hs_align_up(o.strips_bytes, 1024);
    o.spins_bytes = (int64_t)o.rows * o.P * 2;
    o.acc_off = hs_align_up(o.spins_off + o.spins_bytes, 256);
    o.acc_bytes = (int64_t)o.KS * L.ny * o.P * 8;
    o.status_off = hs_align_up(o.acc_off + o.acc_bytes, 256);  // the last 256 bytes: status word first
    o.total = o.status_off + 256;
    return o;
}

}  // namespace

int64_t hs_igemm_scratch(const HsLattice &L, int nsplit) {
    if (nsplit < 1 || nsplit > MAX_SPLIT) return -1;
    return layout_of(L, nsplit).total;
}

// Limit of one pipeline wait of the implicit GEMM (hs_set_wait_limit; WAIT_NS by default).
static unsigned long long g_wait_ns = WAIT_NS;

int hs_set_wait_limit_impl(unsigned long long ns) {
    g_wait_ns = ns ? ns : WAIT_NS;
    return HS_OK;
}

int hs_launch_igemm(const HsLattice &L, int nsplit, void *scratch, int64_t scratch_bytes, cudaStream_t st) {
    if (nsplit < 1 || nsplit > MAX_SPLIT) { hs_set_error("hs_dipolar_full_igemm: nsplit must be 1..3"); return HS_EINVAL; }
    if (!(L.dip_wy == L.ny - 1 && L.dip_wx == L.nx - 1 && !L.dip_wrap)) {
        hs_set_error("hs_dipolar_full_igemm: needs the full (uncropped) kernel; use the direct sum for cut-off windows");
        return HS_EINVAL;
    }
    if (L.ny > 65535 || L.nx > 65535) { hs_set_error("hs_dipolar_full_igemm: lattice too large"); return HS_ERANGE; }
    const Layout lo = layout_of(L, nsplit);
    if (scratch_bytes < lo.total) {
        hs_set_error("hs_dipolar_full_igemm: scratch %lld < %lld bytes", (long long)scratch_bytes, (long long)lo.total);
        return HS_ENOMEM;
    }
    char *base = reinterpret_cast<char *>(scratch);
    __nv_bfloat16 *strips = reinterpret_cast<__nv_bfloat16 *>(base);
    __nv_bfloat16 *spins = reinterpret_cast<__nv_bfloat16 *>(base + lo.spins_off);
    double *acc = reinterpret_cast<double *>(base + lo.acc_off);
    int *status = reinterpret_cast<int *>(base + lo.status_off);
    unsigned long long *first = reinterpret_cast<unsigned long long *>(base + lo.status_off + 8);
    cudaMemsetAsync(status, 0, sizeof(int), st);
    cudaMemsetAsync(first, 0xFF, sizeof(unsigned long long), st);
    first_spin_kernel<<<148 * 4, 256, 0, st>>>(L.m, (int64_t)L.nx * L.ny, first);
    int rc = hs_check_launch("first_spin_kernel");
    if (rc) return rc;
    // near offsets go to the FP64 finalize when the periodic near window does not overlap itself
    const int near_w = (L.nx >= 2 * NEAR_W + 1 && L.ny >= 2 * NEAR_W + 1) ? NEAR_W : -1;
    const int pbc = L.pbc ? 1 : 0;
    const int strip_rows = L.n_sub * (2 * L.ny - 1);
    strips_kernel<<<strip_rows, 256, 0, st>>>(L.K, L.nx, L.ny, L.n_sub, nsplit, lo.qspan, lo.qmin, pbc, near_w, strips);
    if ((rc = hs_check_launch("strips_kernel"))) return rc;
    // the moment must be uniform (the spins are the exact BF16 operand): spins_bf16_kernel flags it
    spins_bf16_kernel<<<148 * 4, 256, 0, st>>>(L.m, L.moment, L.nx, L.ny, lo.P, lo.rows, first, spins, status);
    if ((rc = hs_check_launch("spins_bf16_kernel"))) return rc;
    cudaError_t e = cudaFuncSetAttribute(igemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    if (e != cudaSuccess) { hs_set_error("igemm smem attribute: %s", cudaGetErrorString(e)); return HS_ECUDA; }

    const int grid = lo.XT * lo.YT * lo.KS;
    for (int pass = 0; pass < (L.use_perp ? 2 : 1); ++pass) {
        double *out = pass == 0 ? L.E_dip : L.E_dip_perp;
        const float *Kpass = pass == 0 ? L.K : L.Kps;
        if (pass == 1) {  // perpendicular energy: perp-self kernels
            strips_kernel<<<strip_rows, 256, 0, st>>>(Kpass, L.nx, L.ny, L.n_sub, nsplit, lo.qspan, lo.qmin, pbc, near_w, strips);
            if ((rc = hs_check_launch("strips_kernel"))) return rc;
        }
        cudaMemsetAsync(out, 0, sizeof(double) * (size_t)L.nx * L.ny, st);
        for (int s = 0; s < L.n_sub; ++s) {
            IgemmParams p{strips, spins, lo.qspan, lo.qmin, nsplit, s, lo.P, lo.C, L.nx, L.ny, lo.rows, lo.XT, lo.KS, lo.G, acc, status,
                          g_wait_ns};
            igemm_kernel<<<grid, NT, SMEM_BYTES, st>>>(p);
            if ((rc = hs_check_launch("igemm_kernel"))) return rc;
            igemm_finalize_kernel<<<148 * 4, 256, 0, st>>>(acc, lo.KS, lo.P, L.nx, L.ny, L.ux, L.uy, L.sub_of, s, L.m, L.moment,
                                                           first, Kpass, pbc, near_w, L.dip_pref, out);
            if ((rc = hs_check_launch("igemm_finalize_kernel"))) return rc;
        }
    }
    return HS_OK;
}
