// In-step diagnostics on the device, accumulated in FP64.
//
// The reference computes its segregation diagnostics on the host after a
// device-to-host copy of every position:
//   * segregation(): |COM+ - COM-| / L with plain (non-periodic) means of the
//     positions (src/nbody_gpu_twopass.rs:5364-5393);
//   * compute_segregation_metrics(): NGP counts n+ / n- on an n_cells^3 grid
//     (cell index ((x + L/2) mod L) / cell, in f64), then
//     Var(n+ - n-) / (mean+ + mean-), Corr(delta+, delta-) and the excess
//     variance of n- (src/bin/janus_mu19_production.rs:219-276).
// Here both run on the device over the resident state (no copy of the
// particles), with FP64 accumulation, together with each species' kinetic
// energy (1/2) sum m v^2, momentum sum m v and mean position.
#include "jt_batch.h"

#include <cstring>

namespace {

constexpr int kThreads = 256;

// sums: per species s (0, 1): [0..2] sum x, [3..5] sum m v, [6] sum m v^2 / 2
__global__ void k_diag_particles(const float4* __restrict__ pos, const float4* __restrict__ vel, int64_t n,
                                 float mass, int s, double L, int nc, int* __restrict__ counts,
                                 double* __restrict__ sums)
{
    __shared__ double red[7][kThreads / 32];
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    const double cell = L / nc, half = 0.5 * L;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const float4 p = pos[i], u = vel[i];
        v[0] += p.x;
        v[1] += p.y;
        v[2] += p.z;
        v[3] += (double)mass * u.x;
        v[4] += (double)mass * u.y;
        v[5] += (double)mass * u.z;
        v[6] += 0.5 * (double)mass * ((double)u.x * u.x + (double)u.y * u.y + (double)u.z * u.z);
        // NGP cell as compute_segregation_metrics: rem_euclid then truncate
        double xs[3] = {p.x + half, p.y + half, p.z + half};
        int ic[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            double r = fmod(xs[d], L);
            if (r < 0) r += L;
            long long c = (long long)(r / cell);
            ic[d] = (int)(c % nc);
        }
        atomicAdd(counts + ((int64_t)ic[0] * nc + ic[1]) * nc + ic[2], 1);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 7; k++) {
        double x = v[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) red[k][w] = x;
    }
    __syncthreads();
    if (threadIdx.x < 7) {
        double x = 0;
        for (int j = 0; j < kThreads / 32; j++) x += red[threadIdx.x][j];
        atomicAdd(sums + 7 * s + threadIdx.x, x);
    }
}

// grid sums: [0] sum (d - (mean+ - mean-))^2, d = n+ - n-; [1] sum delta+;
// [2] sum delta-; [3] sum delta+^2; [4] sum delta-^2; [5] sum delta+ delta-;
// [6] sum (n- - mean-)^2
__global__ void k_diag_grid(const int* __restrict__ cp, const int* __restrict__ cm, int64_t ncell,
                            double mean_p, double mean_m, double* __restrict__ sums)
{
    __shared__ double red[7][kThreads / 32];
    double v[7] = {0, 0, 0, 0, 0, 0, 0};
    const double expected = mean_p - mean_m;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ncell;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double a = cp[i], b = cm[i];
        const double d = (a - b) - expected;
        const double dp = mean_p > 0 ? (a - mean_p) / mean_p : 0.0;
        const double dm = mean_m > 0 ? (b - mean_m) / mean_m : 0.0;
        v[0] += d * d;
        v[1] += dp;
        v[2] += dm;
        v[3] += dp * dp;
        v[4] += dm * dm;
        v[5] += dp * dm;
        v[6] += (b - mean_m) * (b - mean_m);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 7; k++) {
        double x = v[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) red[k][w] = x;
    }
    __syncthreads();
    if (threadIdx.x < 7) {
        double x = 0;
        for (int j = 0; j < kThreads / 32; j++) x += red[threadIdx.x][j];
        atomicAdd(sums + threadIdx.x, x);
    }
}

}  // namespace

// Diagnostics of one state (both species) on stream st; scratch is
// allocated and freed here (a diagnostic, not a per-step path).
int jt_diag_state(const float4* const pos[2], const float4* const vel[2], const int64_t n[2],
                  const float mass[2], double L, int n_cells, cudaStream_t st, jt_diag* out)
{
    if (!out || n_cells < 1 || n_cells > 1024 || !(L > 0.0)) return JT_EINVAL;
    const int64_t ncell = (int64_t)n_cells * n_cells * n_cells;
    int* counts = nullptr;
    double* sums = nullptr;
    if (cudaMalloc(&counts, sizeof(int) * 2 * ncell) != cudaSuccess) return JT_ENOMEM;
    if (cudaMalloc(&sums, sizeof(double) * 21) != cudaSuccess) {
        cudaFree(counts);
        return JT_ENOMEM;
    }
    int r = JT_OK;
    if (cudaMemsetAsync(counts, 0, sizeof(int) * 2 * ncell, st) != cudaSuccess ||
        cudaMemsetAsync(sums, 0, sizeof(double) * 21, st) != cudaSuccess)
        r = JT_ECUDA;
    for (int s = 0; s < 2 && r == JT_OK; s++) {
        if (n[s] == 0) continue;
        const unsigned g = (unsigned)std::min<int64_t>((n[s] + kThreads - 1) / kThreads, 148 * 16);
        k_diag_particles<<<g, kThreads, 0, st>>>(pos[s], vel[s], n[s], mass[s], s, L, n_cells,
                                                 counts + s * ncell, sums);
    }
    const double mean_p = (double)n[0] / ncell, mean_m = (double)n[1] / ncell;
    if (r == JT_OK) {
        const unsigned g = (unsigned)std::min<int64_t>((ncell + kThreads - 1) / kThreads, 148 * 16);
        k_diag_grid<<<g, kThreads, 0, st>>>(counts, counts + ncell, ncell, mean_p, mean_m, sums + 14);
    }
    double h[21] = {0};
    if (r == JT_OK && (cudaMemcpyAsync(h, sums, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                       cudaStreamSynchronize(st) != cudaSuccess))
        r = JT_ECUDA;
    cudaFree(counts);
    cudaFree(sums);
    if (r != JT_OK) return r;
    jt_diag d;
    std::memset(&d, 0, sizeof(d));
    for (int s = 0; s < 2; s++) {
        const double* q = h + 7 * s;
        for (int k = 0; k < 3; k++) {
            d.com[s][k] = n[s] > 0 ? q[k] / (double)n[s] : 0.0;
            d.momentum[s][k] = q[3 + k];
        }
        d.kinetic[s] = q[6];
    }
    const double dx = d.com[0][0] - d.com[1][0], dy = d.com[0][1] - d.com[1][1], dz = d.com[0][2] - d.com[1][2];
    d.segregation = std::sqrt(dx * dx + dy * dy + dz * dz) / L;
    const double* gsum = h + 14;
    const double N = (double)ncell;
    const double pois = mean_p + mean_m;
    d.diff_over_poisson = pois > 0 ? (gsum[0] / N) / pois : 0.0;
    const double var_p = gsum[3] / N - (gsum[1] / N) * (gsum[1] / N);
    const double var_m = gsum[4] / N - (gsum[2] / N) * (gsum[2] / N);
    const double cov = gsum[5] / N - (gsum[1] / N) * (gsum[2] / N);
    d.corr = (var_p > 0 && var_m > 0) ? cov / (std::sqrt(var_p) * std::sqrt(var_m)) : 0.0;
    d.exc_var_minus = mean_m > 0 ? ((gsum[6] / N) - mean_m) / mean_m : 0.0;
    *out = d;
    return JT_OK;
}

extern "C" int jt_batch_diagnostics(jt_batch* B, int box_id, int n_cells, jt_diag* out)
{
    jt_box_state* b = jtb_box(B, box_id);
    if (!b) return JT_EINVAL;
    const float4* pos[2] = {b->pos[0], b->pos[1]};
    const float4* vel[2] = {b->vel[0], b->vel[1]};
    return jt_diag_state(pos, vel, b->n, b->mass, b->cfg.box_L, n_cells, jtb_stream(B), out);
}
