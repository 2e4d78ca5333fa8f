/*
 * FP64 periodic force oracle on the GPU.  TEST INFRASTRUCTURE ONLY: the
 * engine (janus-sim_b200/) never links or calls it; tests/ use it to check
 * the engine's accelerations at the production sizes (tens of millions of
 * sources), where the CPU oracle (ewald.c) would take hours.
 *
 * Sources: n particles with FP32 positions (the engine's own inputs, taken
 * exactly) and FP64 charges q_j = s_j m_j (G folded in).  Targets: nt of the
 * sources (by index).  Janus pair rule (janus-sim src/lib.rs:94-121): the
 * acceleration of target i is s_i sum_j q_j (x_j - x_i) K(r).
 *
 * Two outputs per target, both FP64 throughout:
 *
 *   full  = the periodic sum with Plummer softening, as an Ewald sum with a
 *           wide split r_e (independent of the engine's r_s):
 *             reciprocal: s_i sum_{k != 0} (4 pi / V) e^{-k^2 r_e^2} / k^2
 *                           k Im( e^{-i k.x_i} S(k) ),  S(k) = sum_j q_j e^{i k.x_j}
 *             real:       s_i sum_j q_j d S_e(r_p) / r_p^3,  r_p^2 = r^2 + eps^2,
 *                           S_e(r) = erfc(r / 2r_e) + r / (r_e sqrt(pi)) e^{-r^2 / 4r_e^2}
 *           (the same formula as orc_ewald_forces with r_s = r_e; for r << r_e
 *           the real kernel is the softened Newtonian one);
 *
 *   split = the engine's truncated split model at r_s and r_cut: the
 *           Gaussian-filtered Newtonian long part at r_s plus the softened
 *           short part cut at r_cut.  The long part at r_s is obtained from
 *           the Ewald identity for the Newtonian kernel
 *             long(r_s) = long(r_e) + sum_j q_j d [S_e(r) - S_s(r)] / r^3,
 *           so one reciprocal sum serves both outputs:
 *             split = long(r_e) + s_i sum_j q_j d ( [S_e(r) - S_s(r)] / r^3
 *                                              + [r < r_cut] S_s(r_p) / r_p^3 ).
 *           It equals orc_ewald_forces(r_s, eps, r_trunc = r_cut).
 *
 * The real-space sums run over the minimum image within R = 11 r_e
 * (S_e(R) < 1e-12), which must stay below L/2; the reciprocal sum stops at
 * k r_e = sqrt(-ln tol).  Targets are processed in a Morton order so that a
 * warp's targets accept nearly the same sources.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <numeric>
#include <vector>

namespace {

constexpr int kRealThreads = 256;
constexpr int kTile = 256;
constexpr int kModeThreads = 256;

struct RealParams {
    double L, halfL, R2, rc2, eps2;
    double ce, cs;          // 1 / (2 r_e), 1 / (2 r_s)
    double ae, as;          // 1 / (r_e sqrt(pi)), 1 / (r_s sqrt(pi))
    double Rs2;             // (11 r_s)^2: S_s below 1e-12 beyond
    double qm[2];           // charge of species 0 / 1
};

// S(r) for the split scale with c = 1/(2 r_x), a = 1/(r_x sqrt(pi))
__device__ __forceinline__ double split_S(double r, double c, double a)
{
    const double x = r * c;
    return erfc(x) + r * a * exp(-x * x);
}

__device__ __forceinline__ double min_image(double d, double L, double halfL)
{
    if (d > halfL) d -= L;
    else if (d < -halfL) d += L;
    return d;
}

// One block: kRealThreads targets (one per thread) against the sources of
// chunk blockIdx.y; partial sums are added to out_full / out_split.
__global__ void __launch_bounds__(kRealThreads) k_real(const float4* __restrict__ src, int64_t n,
                                                       int64_t chunk, const int64_t* __restrict__ tidx,
                                                       int64_t nt, RealParams P, double* __restrict__ out_full,
                                                       double* __restrict__ out_split)
{
    __shared__ float4 tile[kTile];
    const int64_t t = (int64_t)blockIdx.x * kRealThreads + threadIdx.x;
    const bool tv = t < nt;
    const int64_t ti = tv ? tidx[t] : -1;
    float4 tp = make_float4(0.f, 0.f, 0.f, 0.f);
    if (tv) tp = src[ti];
    const double tx = tp.x, ty = tp.y, tz = tp.z;
    double fx = 0, fy = 0, fz = 0, sx = 0, sy = 0, sz = 0;
    const int64_t j0 = (int64_t)blockIdx.y * chunk;
    const int64_t j1 = min(n, j0 + chunk);
    for (int64_t base = j0; base < j1; base += kTile) {
        const int cnt = (int)(j1 - base < kTile ? j1 - base : kTile);
        __syncthreads();
        if (threadIdx.x < cnt) tile[threadIdx.x] = src[base + threadIdx.x];
        __syncthreads();
        if (!tv) continue;
        for (int jj = 0; jj < cnt; jj++) {
            const float4 s = tile[jj];
            const int64_t j = base + jj;
            const double dx = min_image((double)s.x - tx, P.L, P.halfL);
            const double dy = min_image((double)s.y - ty, P.L, P.halfL);
            const double dz = min_image((double)s.z - tz, P.L, P.halfL);
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 >= P.R2 || j == ti) continue;
            const double q = P.qm[s.w != 0.0f ? 1 : 0];
            const double r = sqrt(r2);
            const double rp2 = r2 + P.eps2;
            const double rp = sqrt(rp2);
            const double Se_p = split_S(rp, P.ce, P.ae);
            const double Se = split_S(r, P.ce, P.ae);
            const double gf = q * Se_p / (rp2 * rp);
            double gs = q * Se / (r2 * r);
            if (r2 < P.Rs2) gs -= q * split_S(r, P.cs, P.as) / (r2 * r);
            if (r2 < P.rc2) gs += q * split_S(rp, P.cs, P.as) / (rp2 * rp);
            fx += gf * dx; fy += gf * dy; fz += gf * dz;
            sx += gs * dx; sy += gs * dy; sz += gs * dz;
        }
    }
    if (tv) {
        atomicAdd(out_full + 3 * t, fx);
        atomicAdd(out_full + 3 * t + 1, fy);
        atomicAdd(out_full + 3 * t + 2, fz);
        atomicAdd(out_split + 3 * t, sx);
        atomicAdd(out_split + 3 * t + 1, sy);
        atomicAdd(out_split + 3 * t + 2, sz);
    }
}

// Structure factors: one thread per mode (half space), sources of chunk
// blockIdx.y; S[2k], S[2k+1] += sum_j q_j (cos, sin)(k.x_j).
__global__ void __launch_bounds__(kModeThreads) k_sfac(const float4* __restrict__ src, int64_t n, int64_t chunk,
                                                       const int4* __restrict__ kv, int64_t nk, double twoL,
                                                       double q0, double q1, double* __restrict__ S)
{
    __shared__ float4 tile[kTile];
    const int64_t k = (int64_t)blockIdx.x * kModeThreads + threadIdx.x;
    const bool kvld = k < nk;
    int4 m = make_int4(0, 0, 0, 0);
    if (kvld) m = kv[k];
    // phase in units of pi: 2 (n . x) / L
    const double ax = m.x * twoL, ay = m.y * twoL, az = m.z * twoL;
    double sr = 0, si = 0;
    const int64_t j0 = (int64_t)blockIdx.y * chunk;
    const int64_t j1 = min(n, j0 + chunk);
    for (int64_t base = j0; base < j1; base += kTile) {
        const int cnt = (int)(j1 - base < kTile ? j1 - base : kTile);
        __syncthreads();
        if (threadIdx.x < cnt) tile[threadIdx.x] = src[base + threadIdx.x];
        __syncthreads();
        if (!kvld) continue;
        for (int jj = 0; jj < cnt; jj++) {
            const float4 s = tile[jj];
            const double ph = ax * (double)s.x + ay * (double)s.y + az * (double)s.z;
            double sn, cs;
            sincospi(ph, &sn, &cs);
            const double q = s.w != 0.0f ? q1 : q0;
            sr += q * cs;
            si += q * sn;
        }
    }
    if (kvld) {
        atomicAdd(S + 2 * k, sr);
        atomicAdd(S + 2 * k + 1, si);
    }
}

// Reciprocal acceleration of each target (without its sign):
// sum_k w_k k Im(conj(e^{i k.x}) S(k)).
__global__ void k_recip_targets(const float4* __restrict__ src, const int64_t* __restrict__ tidx, int64_t nt,
                                const int4* __restrict__ kv, const double* __restrict__ kw, int64_t nk,
                                const double* __restrict__ S, double twoL, double dk, double* __restrict__ out)
{
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nt) return;
    const float4 p = src[tidx[t]];
    double a0 = 0, a1 = 0, a2 = 0;
    for (int64_t k = 0; k < nk; k++) {
        const int4 m = kv[k];
        const double ph = twoL * (m.x * (double)p.x + m.y * (double)p.y + m.z * (double)p.z);
        double sn, cs;
        sincospi(ph, &sn, &cs);
        const double im = cs * S[2 * k + 1] - sn * S[2 * k];
        const double f = kw[k] * im;
        a0 += f * (dk * m.x);
        a1 += f * (dk * m.y);
        a2 += f * (dk * m.z);
    }
    out[3 * t] = a0;
    out[3 * t + 1] = a1;
    out[3 * t + 2] = a2;
}

uint32_t spread3(uint32_t x)
{
    x &= 0x3FF;
    x = (x | (x << 16)) & 0x030000FF;
    x = (x | (x << 8)) & 0x0300F00F;
    x = (x | (x << 4)) & 0x030C30C3;
    x = (x | (x << 2)) & 0x09249249;
    return x;
}

}  // namespace

extern "C" {

/*
 * pos: n x 3 float (host), species: n bytes (0: charge q0, 1: charge q1),
 * tgt: nt source indices (host).  full, split: nt x 3 doubles (host; split
 * may be NULL).  r_e: Ewald split of `full` (R = 11 r_e must be < L/2);
 * r_s, r_cut: the split model of `split`; kcut_tol: reciprocal cut
 * e^{-k^2 r_e^2} >= tol.  Returns 0, or -1 on a bad argument, -2 on a CUDA
 * error.  Allocates its own device memory.
 */
int oge_periodic_forces(const float* pos, const uint8_t* species, int64_t n, double q0, double q1,
                        const int64_t* tgt, int64_t nt, double box, double eps, double r_e, double r_s,
                        double r_cut, double kcut_tol, double* full, double* split)
{
    if (!pos || !species || !tgt || !full || n <= 0 || nt <= 0) return -1;
    if (!(box > 0) || !(r_e > 0) || !(r_s > 0) || !(r_cut > 0) || !(kcut_tol > 0 && kcut_tol < 1)) return -1;
    const double R = 11.0 * r_e;
    if (R >= 0.5 * box || 11.0 * r_s > R || r_cut > R) return -1;
    for (int64_t t = 0; t < nt; t++)
        if (tgt[t] < 0 || tgt[t] >= n) return -1;

    // targets in Morton order of their positions (coherent warps)
    std::vector<int64_t> order(nt);
    std::iota(order.begin(), order.end(), 0);
    std::vector<uint32_t> key(nt);
    for (int64_t t = 0; t < nt; t++) {
        uint32_t c[3];
        for (int d = 0; d < 3; d++) {
            double g = (pos[3 * tgt[t] + d] / box + 0.5) * 1024.0;
            c[d] = (uint32_t)std::min(1023.0, std::max(0.0, g));
        }
        key[t] = spread3(c[0]) | (spread3(c[1]) << 1) | (spread3(c[2]) << 2);
    }
    std::stable_sort(order.begin(), order.end(), [&](int64_t a, int64_t b) { return key[a] < key[b]; });
    std::vector<int64_t> tsorted(nt);
    for (int64_t t = 0; t < nt; t++) tsorted[t] = tgt[order[t]];

    // k vectors of the half space, weights 2 (4 pi / V) e^{-k^2 r_e^2} / k^2
    const double dk = 2.0 * M_PI / box;
    const double kmax = std::sqrt(-std::log(kcut_tol)) / r_e;
    int nmax = (int)std::floor(kmax / dk);
    if (nmax < 1) nmax = 1;
    const double V = box * box * box;
    std::vector<int4> kv;
    std::vector<double> kw;
    for (int nx = 0; nx <= nmax; nx++)
        for (int ny = -nmax; ny <= nmax; ny++)
            for (int nz = -nmax; nz <= nmax; nz++) {
                if (nx == 0 && (ny < 0 || (ny == 0 && nz <= 0))) continue;
                const double k2 = dk * dk * (double)(nx * nx + ny * ny + nz * nz);
                if (k2 > kmax * kmax) continue;
                kv.push_back(make_int4(nx, ny, nz, 0));
                kw.push_back(2.0 * (4.0 * M_PI / V) * std::exp(-k2 * r_e * r_e) / k2);
            }
    const int64_t nk = (int64_t)kv.size();

    std::vector<float4> h_src(n);
    for (int64_t j = 0; j < n; j++)
        h_src[j] = make_float4(pos[3 * j], pos[3 * j + 1], pos[3 * j + 2], species[j] ? 1.0f : 0.0f);

    float4* d_src = nullptr;
    int64_t* d_t = nullptr;
    int4* d_kv = nullptr;
    double *d_kw = nullptr, *d_S = nullptr, *d_rec = nullptr, *d_full = nullptr, *d_split = nullptr;
    int rc = 0;
    auto ok = [&](cudaError_t e) {
        if (e != cudaSuccess && rc == 0) rc = -2;
        return rc == 0;
    };
    ok(cudaMalloc(&d_src, sizeof(float4) * n));
    ok(cudaMalloc(&d_t, sizeof(int64_t) * nt));
    ok(cudaMalloc(&d_kv, sizeof(int4) * nk));
    ok(cudaMalloc(&d_kw, sizeof(double) * nk));
    ok(cudaMalloc(&d_S, sizeof(double) * 2 * nk));
    ok(cudaMalloc(&d_rec, sizeof(double) * 3 * nt));
    ok(cudaMalloc(&d_full, sizeof(double) * 3 * nt));
    ok(cudaMalloc(&d_split, sizeof(double) * 3 * nt));
    if (rc == 0) {
        ok(cudaMemcpy(d_src, h_src.data(), sizeof(float4) * n, cudaMemcpyHostToDevice));
        ok(cudaMemcpy(d_t, tsorted.data(), sizeof(int64_t) * nt, cudaMemcpyHostToDevice));
        ok(cudaMemcpy(d_kv, kv.data(), sizeof(int4) * nk, cudaMemcpyHostToDevice));
        ok(cudaMemcpy(d_kw, kw.data(), sizeof(double) * nk, cudaMemcpyHostToDevice));
        ok(cudaMemset(d_S, 0, sizeof(double) * 2 * nk));
        ok(cudaMemset(d_full, 0, sizeof(double) * 3 * nt));
        ok(cudaMemset(d_split, 0, sizeof(double) * 3 * nt));
    }
    if (rc == 0) {
        const double twoL = 2.0 / box;
        // structure factors: ~2^20 sources per chunk
        const int64_t chunk = 1 << 20;
        dim3 gs((unsigned)((nk + kModeThreads - 1) / kModeThreads), (unsigned)((n + chunk - 1) / chunk));
        k_sfac<<<gs, kModeThreads>>>(d_src, n, chunk, d_kv, nk, twoL, q0, q1, d_S);
        k_recip_targets<<<(unsigned)((nt + 127) / 128), 128>>>(d_src, d_t, nt, d_kv, d_kw, nk, d_S, twoL, dk,
                                                               d_rec);
        RealParams P;
        P.L = box;
        P.halfL = 0.5 * box;
        P.R2 = R * R;
        P.rc2 = r_cut * r_cut;
        P.eps2 = eps * eps;
        P.ce = 1.0 / (2.0 * r_e);
        P.cs = 1.0 / (2.0 * r_s);
        P.ae = 1.0 / (r_e * std::sqrt(M_PI));
        P.as = 1.0 / (r_s * std::sqrt(M_PI));
        P.Rs2 = (11.0 * r_s) * (11.0 * r_s);
        P.qm[0] = q0;
        P.qm[1] = q1;
        // enough blocks for every SM: split the sources into chunks
        const int64_t tblocks = (nt + kRealThreads - 1) / kRealThreads;
        int64_t nchunk = std::max<int64_t>(1, (148 * 8 + tblocks - 1) / tblocks);
        nchunk = std::min<int64_t>(nchunk, std::max<int64_t>(1, n / kTile));
        const int64_t rchunk = (n + nchunk - 1) / nchunk;
        dim3 gr((unsigned)tblocks, (unsigned)nchunk);
        k_real<<<gr, kRealThreads>>>(d_src, n, rchunk, d_t, nt, P, d_full, d_split);
        ok(cudaGetLastError());
        ok(cudaDeviceSynchronize());
    }
    if (rc == 0) {
        std::vector<double> rec(3 * nt), fr(3 * nt), sp(3 * nt);
        ok(cudaMemcpy(rec.data(), d_rec, sizeof(double) * 3 * nt, cudaMemcpyDeviceToHost));
        ok(cudaMemcpy(fr.data(), d_full, sizeof(double) * 3 * nt, cudaMemcpyDeviceToHost));
        ok(cudaMemcpy(sp.data(), d_split, sizeof(double) * 3 * nt, cudaMemcpyDeviceToHost));
        if (rc == 0) {
            for (int64_t t = 0; t < nt; t++) {
                const int64_t o = order[t];
                const double s = species[tsorted[t]] ? (q1 < 0 ? -1.0 : 1.0) : (q0 < 0 ? -1.0 : 1.0);
                for (int d = 0; d < 3; d++) {
                    full[3 * o + d] = s * (rec[3 * t + d] + fr[3 * t + d]);
                    if (split) split[3 * o + d] = s * (rec[3 * t + d] + sp[3 * t + d]);
                }
            }
        }
    }
    cudaFree(d_src);
    cudaFree(d_t);
    cudaFree(d_kv);
    cudaFree(d_kw);
    cudaFree(d_S);
    cudaFree(d_rec);
    cudaFree(d_full);
    cudaFree(d_split);
    return rc;
}

}  // extern "C"
