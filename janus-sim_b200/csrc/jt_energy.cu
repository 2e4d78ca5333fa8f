// Energy diagnostics on the device, FP64.
//
// The reference computes them on the host after copying every particle back
// (src/nbody_gpu_twopass.rs):
//   * kinetic_energy (:5070-5077): sum over all particles of |v|^2 / 2, unit
//     masses;
//   * potential_energy_binding_sampled (:5081-5181): per species a stride
//     sample of at most n_sample particles (i * (n_s / n_sample) in array
//     order), the same-species pair sum -sum_{i<j} 1 / sqrt(r^2 + eps^2)
//     with plain (non-periodic) differences in f64, scaled by
//     n_s (n_s - 1) / (ns (ns - 1));
//   * virialize_sampled (:5186-5225): velocities times alpha = sqrt(|PE| /
//     (2 KE)) when PE < 0;
//   * energy_drift_pct (src/janus_expansion.rs:529-534).
// Here the pair sums run on the device over the resident state (one thread
// per sampled particle i summing j > i, FP64), and the velocities are scaled
// in place.
#include "jt_batch.h"

#include <cmath>

namespace {

constexpr int kT = 256;

__device__ __forceinline__ double block_sum(double v)
{
    __shared__ double red[kT / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kT / 32; w++) t += red[w];
    return t;
}

// -sum_{i<j} 1/sqrt(r^2 + eps^2) over rows i * stride of pos (AoS float3)
__global__ void k_pe_pairs(const float* __restrict__ pos, int64_t ns, int64_t stride, double eps2,
                           double* __restrict__ out)
{
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < ns; i += (int64_t)gridDim.x * blockDim.x) {
        const float* pi = pos + 3 * i * stride;
        const double x = pi[0], y = pi[1], z = pi[2];
        double e = 0.0;
        for (int64_t j = i + 1; j < ns; j++) {
            const float* pj = pos + 3 * j * stride;
            const double dx = x - (double)pj[0], dy = y - (double)pj[1], dz = z - (double)pj[2];
            e -= 1.0 / sqrt(dx * dx + dy * dy + dz * dz + eps2);
        }
        s += e;
    }
    const double t = block_sum(s);
    if (threadIdx.x == 0) atomicAdd(out, t);
}

// sum |v|^2 / 2 (AoS float3)
__global__ void k_ke(const float* __restrict__ vel, int64_t n, double* __restrict__ out)
{
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double x = vel[3 * i], y = vel[3 * i + 1], z = vel[3 * i + 2];
        s += 0.5 * (x * x + y * y + z * z);
    }
    const double t = block_sum(s);
    if (threadIdx.x == 0) atomicAdd(out, t);
}

unsigned grid_for(int64_t n, int cap) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + kT - 1) / kT, cap)); }

struct Bufs {
    float* p[4] = {};
    double* sums = nullptr;
    ~Bufs()
    {
        for (float* q : p) cudaFree(q);
        cudaFree(sums);
    }
};

// Per-species caller-order state copied on the device; n[2] the counts.
int fetch(jt_handle* h, Bufs& B, size_t n[2])
{
    int r = jt_counts(h, &n[0], &n[1]);
    if (r != JT_OK) return r;
    if (n[0] + n[1] == 0) return JT_ESTATE;
    for (int k = 0; k < 4; k++) {
        const size_t m = n[k / 2];
        if (m && cudaMalloc(&B.p[k], sizeof(float) * 3 * m) != cudaSuccess) {
            cudaGetLastError();
            return JT_ENOMEM;
        }
    }
    if (cudaMalloc(&B.sums, sizeof(double) * 4) != cudaSuccess) {
        cudaGetLastError();
        return JT_ENOMEM;
    }
    return jt_get_state(h, B.p[0], B.p[1], B.p[2], B.p[3], JT_MEM_DEVICE);
}

// sums[0] KE, sums[1] PE+, sums[2] PE- (raw, unscaled)
int energies(const Bufs& B, const size_t n[2], size_t n_sample, double eps2, double* h, size_t ns[2])
{
    if (cudaMemset(B.sums, 0, sizeof(double) * 4) != cudaSuccess) return JT_ECUDA;
    for (int s = 0; s < 2; s++) {
        if (n[s] == 0) {
            ns[s] = 0;
            continue;
        }
        k_ke<<<grid_for((int64_t)n[s], 148 * 8), kT>>>(B.p[2 * s + 1], (int64_t)n[s], B.sums);
        // stride sampling exactly as the reference: all when n <= n_sample
        const size_t stride = n[s] <= n_sample ? 1 : n[s] / n_sample;
        ns[s] = n[s] <= n_sample ? n[s] : n_sample;
        k_pe_pairs<<<grid_for((int64_t)ns[s], 148 * 16), kT>>>(B.p[2 * s], (int64_t)ns[s], (int64_t)stride, eps2,
                                                                B.sums + 1 + s);
    }
    if (cudaGetLastError() != cudaSuccess) return JT_ECUDA;
    if (cudaMemcpy(h, B.sums, sizeof(double) * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return JT_ECUDA;
    return JT_OK;
}

double pair_scale(size_t n, size_t ns)
{
    return ns > 1 ? ((double)n * (double)(n - 1)) / ((double)ns * (double)(ns - 1)) : 1.0;
}

}  // namespace

extern "C" {

int jt_energy_sampled(jt_handle* h, size_t n_sample, jt_energy* out)
{
    if (!h || !out || n_sample < 1) return JT_EINVAL;
    jt_config cfg;
    float mp = 0.f, mm = 0.f;
    int r = jth_info(h, &cfg, &mp, &mm, nullptr);
    if (r != JT_OK) return r;
    Bufs B;
    size_t n[2];
    if ((r = fetch(h, B, n)) != JT_OK) return r;
    double s[4];
    size_t ns[2];
    if ((r = energies(B, n, n_sample, cfg.softening * cfg.softening, s, ns)) != JT_OK) return r;
    out->kinetic = s[0];
    out->pe_plus = s[1] * pair_scale(n[0], ns[0]);
    out->pe_minus = s[2] * pair_scale(n[1], ns[1]);
    out->pe_binding = out->pe_plus + out->pe_minus;
    out->n_sampled[0] = (int64_t)ns[0];
    out->n_sampled[1] = (int64_t)ns[1];
    return JT_OK;
}

int jt_virialize_sampled(jt_handle* h, size_t n_sample, double* alpha)
{
    if (!h || n_sample < 1) return JT_EINVAL;
    jt_energy e;
    int r = jt_energy_sampled(h, n_sample, &e);
    if (r != JT_OK) return r;
    // the reference skips tiny KE and unbound systems (:5190-5200)
    if (e.kinetic < 1e-20 || e.pe_binding >= 0.0) {
        if (alpha) *alpha = 1.0;
        return JT_OK;
    }
    const double a = std::sqrt((std::fabs(e.pe_binding) / 2.0) / e.kinetic);
    if ((r = jth_scale_velocities(h, (float)a)) != JT_OK) return r;
    if (alpha) *alpha = a;
    return JT_OK;
}

double jt_energy_drift_pct(double e_now, double e_initial)
{
    if (std::fabs(e_initial) < 1e-30) return 0.0;
    return (e_now - e_initial) / std::fabs(e_initial) * 100.0;
}

}  // extern "C"
