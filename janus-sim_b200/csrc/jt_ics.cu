// Zel'dovich lattice initial conditions generated on the device.
//
// The workload spec: per species an n^3 lattice (the m- lattice offset by
// half a cell), Zel'dovich displacements psi = i k / k^2 delta(k) of a
// seeded Gaussian random field with P(k) = A k^-2.5 exp(-(k/k_c)^2), k_c =
// half the lattice Nyquist wavenumber, A such that rms |psi+| = rms_frac *
// spacing, and psi- = -psi evaluated on the offset lattice (delta- =
// -delta+).  Velocities are the growing mode v = vel_factor * psi.  This
// replaces the host-side generators (the reference's src/ic_gen.rs:52-176
// builds its ICs on the CPU with rustfft; here the field, the transforms and
// the particle placement stay on the device).
//
// Steps: white noise (Philox4x32-10 counter-based generator, Salmon et al.,
// SC'11, then Box-Muller in FP64) -> cuFFT R2C -> per component and species
// one k-space kernel (amplitude, i k / k^2, the half-cell phase shift for m-)
// and cuFFT C2R -> FP64 sum of |psi+|^2 -> placement.  The Nyquist planes are
// zeroed, so every spectrum handed to C2R is exactly Hermitian.
#include "jt_batch.h"

#include <cufft.h>

#include <cmath>
#include <cstring>

namespace {

// ------------------------------------------------------------ Philox4x32-10
struct P4 {
    unsigned x, y, z, w;
};

__host__ __device__ inline unsigned mulhi32(unsigned a, unsigned b)
{
    return (unsigned)(((unsigned long long)a * b) >> 32);
}

__host__ __device__ inline P4 philox4x32_10(P4 c, unsigned k0, unsigned k1)
{
    const unsigned M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const unsigned W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const unsigned hi0 = mulhi32(M0, c.x), lo0 = M0 * c.x;
        const unsigned hi1 = mulhi32(M1, c.z), lo1 = M1 * c.z;
        c = P4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
        k0 += W0;
        k1 += W1;
    }
    return c;
}

constexpr int kT = 256;

// unit Gaussian per cell: counter (idx lo, idx hi, 0, 0), key = seed;
// u = (r + 0.5) 2^-32, g = sqrt(-2 ln u0) cos(2 pi u1) in FP64
__global__ void k_noise(float* __restrict__ out, int64_t n3, unsigned k0, unsigned k1)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n3) return;
    const P4 r = philox4x32_10(P4{(unsigned)i, (unsigned)((uint64_t)i >> 32), 0u, 0u}, k0, k1);
    const double u0 = ((double)r.x + 0.5) * 2.3283064365386963e-10;
    const double u1 = ((double)r.y + 0.5) * 2.3283064365386963e-10;
    out[i] = (float)(sqrt(-2.0 * log(u0)) * cospi(2.0 * u1));
}

// one displacement component (comp 0 x, 1 y, 2 z) of one species (sp 0 m+,
// 1 m-) from the noise spectrum: psi_k = i k_c / k^2 A(k) delta_k, times
// -exp(i a/2 (kx + ky + kz)) for m-; zero at k = 0 and on the Nyquist planes
__global__ void k_psi(const float2* __restrict__ dk, float2* __restrict__ out, int n, double dkf,
                      double kc, double a, int comp, int sp)
{
    const int nh = n / 2 + 1;
    const int64_t total = (int64_t)n * n * nh;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= total) return;
    const int ix = (int)(i % nh);
    const int iy = (int)((i / nh) % n);
    const int iz = (int)(i / ((int64_t)nh * n));
    const bool nyq = (n % 2 == 0) && (ix == n / 2 || iy == n / 2 || iz == n / 2);
    const double kx = dkf * ix;
    const double ky = dkf * (iy <= (n - 1) / 2 ? iy : iy - n);
    const double kz = dkf * (iz <= (n - 1) / 2 ? iz : iz - n);
    const double k2 = kx * kx + ky * ky + kz * kz;
    if (k2 == 0.0 || nyq) {
        out[i] = make_float2(0.f, 0.f);
        return;
    }
    const double k = sqrt(k2);
    const double amp = pow(k, -1.25) * exp(-0.5 * (k / kc) * (k / kc));
    const double kcmp = comp == 0 ? kx : (comp == 1 ? ky : kz);
    const double f = kcmp / k2 * amp;
    const float2 d = dk[i];
    // i f (dr + i di) = -f di + i f dr
    double re = -f * d.y, im = f * d.x;
    if (sp == 1) {
        double s, c;
        sincos(0.5 * a * (kx + ky + kz), &s, &c);
        const double r2 = re * c - im * s, i2 = re * s + im * c;
        re = -r2;
        im = -i2;
    }
    out[i] = make_float2((float)re, (float)im);
}

// sum of |psi+|^2 over the lattice (FP64)
__global__ void k_sumsq(const float* __restrict__ px, const float* __restrict__ py,
                        const float* __restrict__ pz, int64_t n3, double* __restrict__ out)
{
    __shared__ double red[kT / 32];
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n3; i += (int64_t)gridDim.x * blockDim.x) {
        const double x = px[i], y = py[i], z = pz[i];
        s += x * x + y * y + z * z;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kT / 32; w++) t += red[w];
        atomicAdd(out, t);
    }
}

// lattice point (iz, iy, ix) -> row iz n^2 + iy n + ix: position
// (i + 0.5) a - L/2 (+ a/2 for m-) + scale psi, wrapped into [-L/2, L/2);
// velocity vel_factor scale psi (AoS float3)
__global__ void k_place(const float* __restrict__ px, const float* __restrict__ py,
                        const float* __restrict__ pz, int n, float a, float L, float off,
                        const double* __restrict__ sumsq, double rms_frac, float vel_factor,
                        float* __restrict__ pos, float* __restrict__ vel)
{
    const int64_t n3 = (int64_t)n * n * n;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n3) return;
    const double rms = sqrt(*sumsq / (double)n3);
    const float scale = rms > 0.0 ? (float)(rms_frac * (double)a / rms) : 0.f;
    const int ix = (int)(i % n), iy = (int)((i / n) % n), iz = (int)(i / ((int64_t)n * n));
    const float hL = 0.5f * L;
    const float d[3] = {px[i] * scale, py[i] * scale, pz[i] * scale};
    const int id[3] = {ix, iy, iz};
#pragma unroll
    for (int c = 0; c < 3; c++) {
        float x = ((float)id[c] + 0.5f) * a - hL + off + d[c];
        x = x - L * floorf((x + hL) / L);
        if (x >= hL) x -= L;
        if (x < -hL) x += L;
        pos[3 * i + c] = x;
        if (vel) vel[3 * i + c] = vel_factor * d[c];
    }
}

unsigned blocks(int64_t n) { return (unsigned)((n + kT - 1) / kT); }

struct Scratch {
    float* noise = nullptr;
    float2* spec = nullptr;
    float2* work = nullptr;
    float* psi[6] = {};
    double* sumsq = nullptr;
    cufftHandle r2c = 0, c2r = 0;
    bool have_r2c = false, have_c2r = false;
    ~Scratch()
    {
        if (have_r2c) cufftDestroy(r2c);
        if (have_c2r) cufftDestroy(c2r);
        cudaFree(noise);
        cudaFree(spec);
        cudaFree(work);
        for (float* p : psi) cudaFree(p);
        cudaFree(sumsq);
    }
};

bool valid_params(const jt_ics_params* p)
{
    return p && p->n_side >= 4 && p->n_side <= 1024 && p->box_L > 0.0 && std::isfinite(p->box_L) &&
           p->rms_frac >= 0.0 && std::isfinite(p->rms_frac) && std::isfinite(p->vel_factor);
}

// Generate into device AoS arrays pos_p, vel_p, pos_m, vel_m (n^3 rows each;
// the velocity pointers may be null) on stream st.
int generate(const jt_ics_params* p, float* pos_p, float* vel_p, float* pos_m, float* vel_m, cudaStream_t st)
{
    const int n = p->n_side;
    const int64_t n3 = (int64_t)n * n * n;
    const int64_t nc = (int64_t)n * n * (n / 2 + 1);
    Scratch S;
    if (cudaMalloc(&S.noise, sizeof(float) * n3) != cudaSuccess ||
        cudaMalloc(&S.spec, sizeof(float2) * nc) != cudaSuccess ||
        cudaMalloc(&S.work, sizeof(float2) * nc) != cudaSuccess ||
        cudaMalloc(&S.sumsq, sizeof(double)) != cudaSuccess) {
        cudaGetLastError();
        return JT_ENOMEM;
    }
    for (int c = 0; c < 6; c++)
        if (cudaMalloc(&S.psi[c], sizeof(float) * n3) != cudaSuccess) {
            cudaGetLastError();
            return JT_ENOMEM;
        }
    if (cufftPlan3d(&S.r2c, n, n, n, CUFFT_R2C) != CUFFT_SUCCESS) return JT_ECUDA;
    S.have_r2c = true;
    if (cufftPlan3d(&S.c2r, n, n, n, CUFFT_C2R) != CUFFT_SUCCESS) return JT_ECUDA;
    S.have_c2r = true;
    if (cufftSetStream(S.r2c, st) != CUFFT_SUCCESS || cufftSetStream(S.c2r, st) != CUFFT_SUCCESS)
        return JT_ECUDA;
    const double a = p->box_L / n;
    const double dkf = 2.0 * M_PI / p->box_L;
    const double kc = 0.5 * (M_PI / a);
    k_noise<<<blocks(n3), kT, 0, st>>>(S.noise, n3, (unsigned)p->seed, (unsigned)(p->seed >> 32));
    if (cufftExecR2C(S.r2c, S.noise, (cufftComplex*)S.spec) != CUFFT_SUCCESS) return JT_ECUDA;
    for (int sp = 0; sp < 2; sp++)
        for (int c = 0; c < 3; c++) {
            k_psi<<<blocks(nc), kT, 0, st>>>(S.spec, S.work, n, dkf, kc, a, c, sp);
            if (cufftExecC2R(S.c2r, (cufftComplex*)S.work, S.psi[3 * sp + c]) != CUFFT_SUCCESS)
                return JT_ECUDA;
        }
    if (cudaMemsetAsync(S.sumsq, 0, sizeof(double), st) != cudaSuccess) return JT_ECUDA;
    k_sumsq<<<(unsigned)std::min<int64_t>(blocks(n3), 148 * 8), kT, 0, st>>>(S.psi[0], S.psi[1], S.psi[2], n3,
                                                                              S.sumsq);
    // C2R is unnormalised: both the rms and psi carry the same factor n^3,
    // which the rms normalisation removes
    k_place<<<blocks(n3), kT, 0, st>>>(S.psi[0], S.psi[1], S.psi[2], n, (float)a, (float)p->box_L, 0.f,
                                       S.sumsq, p->rms_frac, (float)p->vel_factor, pos_p, vel_p);
    k_place<<<blocks(n3), kT, 0, st>>>(S.psi[3], S.psi[4], S.psi[5], n, (float)a, (float)p->box_L,
                                       (float)(0.5 * a), S.sumsq, p->rms_frac, (float)p->vel_factor, pos_m,
                                       vel_m);
    if (cudaGetLastError() != cudaSuccess) return JT_ECUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return JT_ECUDA;
    return JT_OK;
}

struct DevBuf {
    float* p[4] = {};
    ~DevBuf()
    {
        for (float* q : p) cudaFree(q);
    }
    int alloc(int64_t n3)
    {
        for (auto& q : p)
            if (cudaMalloc(&q, sizeof(float) * 3 * n3) != cudaSuccess) {
                cudaGetLastError();
                return JT_ENOMEM;
            }
        return JT_OK;
    }
};

}  // namespace

extern "C" {

int jt_ics_zeldovich(const jt_ics_params* p, float* pos_p, float* vel_p, float* pos_m, float* vel_m, int mem)
{
    if (!valid_params(p) || !pos_p || !pos_m || (mem != JT_MEM_HOST && mem != JT_MEM_DEVICE)) return JT_EINVAL;
    const int64_t n3 = (int64_t)p->n_side * p->n_side * p->n_side;
    if (mem == JT_MEM_DEVICE) return generate(p, pos_p, vel_p, pos_m, vel_m, 0);
    DevBuf d;
    int r = d.alloc(n3);
    if (r != JT_OK) return r;
    if ((r = generate(p, d.p[0], d.p[1], d.p[2], d.p[3], 0)) != JT_OK) return r;
    float* host[4] = {pos_p, vel_p, pos_m, vel_m};
    for (int k = 0; k < 4; k++)
        if (host[k] && cudaMemcpy(host[k], d.p[k], sizeof(float) * 3 * n3, cudaMemcpyDeviceToHost) != cudaSuccess)
            return JT_ECUDA;
    return JT_OK;
}

int jt_set_state_zeldovich(jt_handle* h, const jt_ics_params* p)
{
    if (!h || !valid_params(p)) return JT_EINVAL;
    const int64_t n3 = (int64_t)p->n_side * p->n_side * p->n_side;
    DevBuf d;
    int r = d.alloc(n3);
    if (r != JT_OK) return r;
    if ((r = generate(p, d.p[0], d.p[1], d.p[2], d.p[3], 0)) != JT_OK) return r;
    return jt_set_state(h, d.p[0], d.p[1], (size_t)n3, d.p[2], d.p[3], (size_t)n3, JT_MEM_DEVICE);
}

int jt_batch_add_zeldovich(jt_batch* b, const jt_config* cfg, const jt_ics_params* p, int* box_id)
{
    if (!b || !cfg || !box_id || !valid_params(p)) return JT_EINVAL;
    const int64_t n3 = (int64_t)p->n_side * p->n_side * p->n_side;
    DevBuf d;
    int r = d.alloc(n3);
    if (r != JT_OK) return r;
    if ((r = generate(p, d.p[0], d.p[1], d.p[2], d.p[3], 0)) != JT_OK) return r;
    return jt_batch_add(b, cfg, d.p[0], d.p[1], (size_t)n3, d.p[2], d.p[3], (size_t)n3, JT_MEM_DEVICE, box_id);
}

// Philox4x32-10 on the host, for checking the device stream (the
// generator's known-answer vectors)
void jt_philox4x32_10(const unsigned ctr[4], const unsigned key[2], unsigned out[4])
{
    const P4 r = philox4x32_10(P4{ctr[0], ctr[1], ctr[2], ctr[3]}, key[0], key[1]);
    out[0] = r.x;
    out[1] = r.y;
    out[2] = r.z;
    out[3] = r.w;
}

}  // extern "C"
