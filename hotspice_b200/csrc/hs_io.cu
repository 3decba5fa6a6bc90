// Reservoir input / output stepping (hotspice/io.py:193-500) on the device.
//
// The experiments drive a lattice with a sequence of inputs; each input sets a uniform or
// patterned Zeeman field (ZeemanEnergy.set_field, hotspice/energies.py:97-118), runs
// Magnets.progress(t_max, MCsteps_max) (core.py:736-760) and reads a coarse-grained state
// (io.py:312-446). Here each of those is a stream-ordered device operation, so a whole input
// sequence is enqueued without a host round trip:
//   zeeman_field_kernel  E_factor / E_factor_perp of every cell, in place (FP64 and the FP32
//                        copies the step kernels read), from magnitude * pattern and the angle
//   progress_arm_kernel  t0 = t, mc0 = attempted / n, the limits, progress = 1, done = 0: the
//                        persistent engine launch that follows runs until the stop rule holds
//                        (or its step budget is used up, which the next arm / disarm reports
//                        as HS_ST_STEP_CAP)
//   region_sum_kernel    one CTA per output region (a rectangle of cells), FP64 tree sum of
//                        m * weight, divided by the region's normalisation
#include "hs_common.cuh"
#include "hs_internal.h"

namespace {

constexpr int IO_T = 256;

__global__ void __launch_bounds__(IO_T) zeeman_field_kernel(int64_t N, int in_plane, const double *moment,
                                                            const double *orient, const float *pattern, double magnitude,
                                                            double ca, double sa, double *ef, double *efp, float *ef32,
                                                            float *efp32) {
    for (int64_t i = (int64_t)blockIdx.x * IO_T + threadIdx.x; i < N; i += (int64_t)gridDim.x * IO_T) {
        const double mag = pattern ? magnitude * (double)pattern[i] : magnitude;
        double e, ep;
        if (in_plane) {
            const double bx = mag * ca, by = mag * sa;
            const double ox = orient[2 * i], oy = orient[2 * i + 1];
            e = -moment[i] * (bx * ox + by * oy);
            ep = -moment[i] * (by * ox - bx * oy);
        } else {
            e = -moment[i] * mag;
            ep = 0.0;
        }
        if (ef) ef[i] = e;
        if (efp) efp[i] = ep;
        ef32[i] = (float)e;
        if (efp32) efp32[i] = (float)ep;
    }
}

__global__ void progress_arm_kernel(HsCounters *C, int n_occ, double t_max, double mc_max) {
    if (C->progress && !C->done) C->status |= HS_ST_STEP_CAP;   // the previous armed run did not finish
    C->t0 = C->t;
    C->mc0 = (double)C->attempted / (double)n_occ;
    C->t_max = t_max;
    C->mc_max = mc_max;
    C->progress = 1;
    C->done = 0;
}

__global__ void progress_disarm_kernel(HsCounters *C) {
    if (C->progress && !C->done) C->status |= HS_ST_STEP_CAP;
    C->progress = 0;
    C->done = 0;
}

__global__ void __launch_bounds__(IO_T) region_sum_kernel(const int8_t *m, int nx, int ny, int R, const int32_t *rects,
                                                          const double *wx, const double *wy, const double *norm,
                                                          double *out) {
    __shared__ double s_x[IO_T], s_y[IO_T];
    const int r = blockIdx.x;
    // the rectangle [y0, y1) x [x0, x1), clipped to the lattice
    const int y0 = max(rects[4 * r], 0), y1 = min(rects[4 * r + 1], ny);
    const int x0 = max(rects[4 * r + 2], 0), x1 = min(rects[4 * r + 3], nx);
    const int w = x1 - x0;
    const int64_t cells = (y1 > y0 && w > 0) ? (int64_t)(y1 - y0) * w : 0;
    double ax = 0.0, ay = 0.0;
    for (int64_t k = threadIdx.x; k < cells; k += IO_T) {
        const int64_t i = (int64_t)(y0 + (int)(k / w)) * nx + x0 + (int)(k % w);
        const double mi = (double)m[i];
        ax += mi * wx[i];
        if (wy) ay += mi * wy[i];
    }
    s_x[threadIdx.x] = ax;
    s_y[threadIdx.x] = ay;
    __syncthreads();
    for (int o = IO_T / 2; o > 0; o >>= 1) {
        if ((int)threadIdx.x < o) {
            s_x[threadIdx.x] += s_x[threadIdx.x + o];
            s_y[threadIdx.x] += s_y[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[r] = s_x[0] / norm[r];
        if (wy) out[R + r] = s_y[0] / norm[r];
    }
}

// Vertex types of in-plane square ASI (examples/IP_SquareVertices.py:19-35): a vertex is a
// cell with even x and y; with its four neighbours (periodic wrap) N_in = up + left - right -
// down and N_flower = up - left + right - down, the vertex is type 3 / 4 when |N_in| = 2 / 4,
// else type 1 when |N_flower| = 4 and type 2 otherwise. Integer counts, one atomic per warp.
__global__ void __launch_bounds__(IO_T) square_vertex_kernel(const int8_t *m, int nx, int ny, unsigned long long *out) {
    const int vx = (nx + 1) / 2, vy = (ny + 1) / 2;
    const int64_t nv = (int64_t)vx * vy;
    unsigned c[4] = {0u, 0u, 0u, 0u};
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < nv; v += (int64_t)gridDim.x * blockDim.x) {
        const int y = 2 * (int)(v / vx), x = 2 * (int)(v % vx);
        const int yu = y == 0 ? ny - 1 : y - 1, yd = y + 1 == ny ? 0 : y + 1;
        const int xl = x == 0 ? nx - 1 : x - 1, xr = x + 1 == nx ? 0 : x + 1;
        const int up = m[(int64_t)yu * nx + x], down = m[(int64_t)yd * nx + x];
        const int left = m[(int64_t)y * nx + xl], right = m[(int64_t)y * nx + xr];
        const int n_in = abs(up + left - right - down), flower = abs(up - left + right - down);
        const int t = n_in == 4 ? 3 : (n_in == 2 ? 2 : (n_in == 0 ? (flower == 4 ? 0 : 1) : -1));
#pragma unroll
        for (int k = 0; k < 4; ++k) c[k] += (t == k);
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        unsigned s = c[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0 && s) atomicAdd(out + k, (unsigned long long)s);
    }
}

}  // namespace

int hs_square_vertex_counts_impl(const int8_t *m, int nx, int ny, int64_t *out, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(out, 0, 4 * sizeof(int64_t), st);
    if (e != cudaSuccess) { hs_set_error("hs_square_vertex_counts: %s", cudaGetErrorString(e)); return HS_ECUDA; }
    const int64_t nv = (int64_t)((nx + 1) / 2) * ((ny + 1) / 2);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>((nv + IO_T - 1) / IO_T, 148 * 8));
    square_vertex_kernel<<<grid, IO_T, 0, st>>>(m, nx, ny, reinterpret_cast<unsigned long long *>(out));
    return hs_check_launch("square_vertex_kernel");
}

int hs_zeeman_set_impl(int64_t n_cells, int in_plane, const double *moment, const double *orient, const float *pattern,
                       double magnitude, double angle, double *ef, double *efp, float *ef32, float *efp32, cudaStream_t st) {
    const int nb = (int)std::min<int64_t>((n_cells + IO_T - 1) / IO_T, 148 * 16);
    // cos / sin of the angle on the host, as numpy evaluates them for the reference's field
    zeeman_field_kernel<<<std::max(nb, 1), IO_T, 0, st>>>(n_cells, in_plane, moment, orient, pattern, magnitude,
                                                         cos(angle), sin(angle), ef, efp, ef32, efp32);
    return hs_check_launch("zeeman_field_kernel");
}

int hs_progress_arm_impl(HsCounters *C, int n_occ, double t_max, double mc_max, cudaStream_t st) {
    progress_arm_kernel<<<1, 1, 0, st>>>(C, n_occ, t_max, mc_max);
    return hs_check_launch("progress_arm_kernel");
}

int hs_progress_disarm_impl(HsCounters *C, cudaStream_t st) {
    progress_disarm_kernel<<<1, 1, 0, st>>>(C);
    return hs_check_launch("progress_disarm_kernel");
}

int hs_region_readout_impl(const int8_t *m, int nx, int ny, int R, const int32_t *rects, const double *wx,
                           const double *wy, const double *norm, double *out, cudaStream_t st) {
    region_sum_kernel<<<R, IO_T, 0, st>>>(m, nx, ny, R, rects, wx, wy, norm, out);
    return hs_check_launch("region_sum_kernel");
}
