// Particle-mesh kernels: signed CIC deposit and the fused k-space kernel.
//
// Reference: cic_scatter (src/nbody_gpu_twopass.rs:98-158) deposits counts of
// each species into two f64 grids with CAS-loop atomics; cufft_solve_device
// (cuda/cufft_wrapper.cu:350-398) then runs, per species, a D2D copy, D2Z,
// apply_green_kernel (:148-208), Z2D and a normalisation kernel, each followed
// by a device synchronisation.
//
// Here: one FP32 grid holds the signed source rho = sum_j s_j m_j W / h^3 of
// both species (the reference's F+ = -grad phi+ + grad phi- is the same linear
// combination), deposited with native float reductions by particles in Morton
// order; one R2C; ONE k-space kernel applies Green x Gaussian filter (x CIC
// deconvolution x spectral gradient in the accurate mode) and the 1/M^3
// normalisation and writes the three force spectra; one batched C2R (batch 3)
// produces the three force grids.  The compatibility mode writes the potential
// spectrum only (the reference's Green, r_s = r_cut/3, k_min filter) and
// differentiates in real space as the reference does.
#include "jt_internal.cuh"

namespace {

// ---- accurate deposit: nodes at -L/2 + i h, floor-based CIC, wrap by mask
__global__ void k_deposit(const float4* __restrict__ pos0, int64_t n0, float q0,
                          const float4* __restrict__ pos1, int64_t n1, float q1,
                          float* __restrict__ rho, int M, float halfL, float hinv)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n0 + n1) return;
    float4 p;
    float q;
    if (i < n0) { p = pos0[i]; q = q0; } else { p = pos1[i - n0]; q = q1; }
    float gx = (p.x + halfL) * hinv, gy = (p.y + halfL) * hinv, gz = (p.z + halfL) * hinv;
    float fx0 = floorf(gx), fy0 = floorf(gy), fz0 = floorf(gz);
    float fx = gx - fx0, fy = gy - fy0, fz = gz - fz0;
    int mask = M - 1;
    int ix = (int)fx0 & mask, iy = (int)fy0 & mask, iz = (int)fz0 & mask;
    int ix1 = (ix + 1) & mask, iy1 = (iy + 1) & mask, iz1 = (iz + 1) & mask;
    int64_t MM = (int64_t)M * M;
    int64_t r00 = (int64_t)iy * M + (int64_t)iz * MM, r10 = (int64_t)iy1 * M + (int64_t)iz * MM;
    int64_t r01 = (int64_t)iy * M + (int64_t)iz1 * MM, r11 = (int64_t)iy1 * M + (int64_t)iz1 * MM;
    float wx0 = 1.0f - fx, wy0 = 1.0f - fy, wz0 = 1.0f - fz;
    float a00 = q * wy0 * wz0, a10 = q * fy * wz0, a01 = q * wy0 * fz, a11 = q * fy * fz;
    atomicAdd(rho + r00 + ix, a00 * wx0);
    atomicAdd(rho + r00 + ix1, a00 * fx);
    atomicAdd(rho + r10 + ix, a10 * wx0);
    atomicAdd(rho + r10 + ix1, a10 * fx);
    atomicAdd(rho + r01 + ix, a01 * wx0);
    atomicAdd(rho + r01 + ix1, a01 * fx);
    atomicAdd(rho + r11 + ix, a11 * wx0);
    atomicAdd(rho + r11 + ix1, a11 * fx);
}

// ---- compatibility deposit: the reference's coordinates and weights
// (fmodf wrap, (int) truncation, weight wx*wy*wz in float), signed mass
__global__ void k_deposit_rc(const float4* __restrict__ pos, const int8_t* __restrict__ sg,
                             int64_t n, float m0, float m1, float* __restrict__ rho, int M,
                             float box_half, float inv_cell, float inv_vol)
{
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    float4 p = pos[t];
    float gx = __fmul_rn(__fadd_rn(p.x, box_half), inv_cell);
    float gy = __fmul_rn(__fadd_rn(p.y, box_half), inv_cell);
    float gz = __fmul_rn(__fadd_rn(p.z, box_half), inv_cell);
    float Mf = (float)M;
    gx = fmodf(__fadd_rn(gx, Mf), Mf);
    gy = fmodf(__fadd_rn(gy, Mf), Mf);
    gz = fmodf(__fadd_rn(gz, Mf), Mf);
    int ix = (int)gx, iy = (int)gy, iz = (int)gz;
    float fx = __fsub_rn(gx, (float)ix), fy = __fsub_rn(gy, (float)iy), fz = __fsub_rn(gz, (float)iz);
    float wx[2] = {__fsub_rn(1.0f, fx), fx}, wy[2] = {__fsub_rn(1.0f, fy), fy},
          wz[2] = {__fsub_rn(1.0f, fz), fz};
    // positions outside the box (or NaN) still index inside the grid
    ix = ((ix % M) + M) % M; iy = ((iy % M) + M) % M; iz = ((iz % M) + M) % M;
    float q = (sg[t] > 0 ? m0 : -m1) * inv_vol;
#pragma unroll
    for (int di = 0; di < 2; di++)
#pragma unroll
        for (int dj = 0; dj < 2; dj++)
#pragma unroll
            for (int dk = 0; dk < 2; dk++) {
                int ci = (ix + di) % M, cj = (iy + dj) % M, ck = (iz + dk) % M;
                float w = __fmul_rn(__fmul_rn(wx[di], wy[dj]), wz[dk]);
                atomicAdd(rho + ci + (int64_t)M * (cj + (int64_t)M * ck), w * q);
            }
}

// per-axis factors of the accurate Green's function (separable):
//   ax[n] = { k_n, grad factor (0 at Nyquist), exp(-k_n^2 r_s^2) / sinc^4(pi n / M), |n| }
__global__ void k_kspace_acc(const float2* __restrict__ rho_k, float2* __restrict__ out, int M,
                             const float4* __restrict__ axis, float norm, int k_min,
                             int64_t Gc)
{
    int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= Gc) return;
    int Mh = M / 2 + 1;
    int kx = (int)(idx % Mh);
    int64_t r = idx / Mh;
    int ky = (int)(r % M);
    int kz = (int)(r / M);
    float4 ax = __ldg(&axis[kx]), ay = __ldg(&axis[ky]), az = __ldg(&axis[kz]);
    float k2 = ax.x * ax.x + ay.x * ay.x + az.x * az.x;
    int kmax = max(max((int)ax.w, (int)ay.w), (int)az.w);
    float2 z = rho_k[idx];
    float2 o0 = make_float2(0.f, 0.f), o1 = o0, o2 = o0;
    if (k2 > 0.0f && kmax >= k_min) {
        // -4 pi / k^2 * filter * deconvolution * 1/M^3
        float green = -12.566370614f * norm * (ax.z * ay.z * az.z) / k2;
        float pr = z.x * green, pi = z.y * green;
        // a_d(k) = -i k_d phi(k) = k_d (pi, -pr)
        o0 = make_float2(ax.y * pi, -ax.y * pr);
        o1 = make_float2(ay.y * pi, -ay.y * pr);
        o2 = make_float2(az.y * pi, -az.y * pr);
    }
    out[idx] = o0;
    out[Gc + idx] = o1;
    out[2 * Gc + idx] = o2;
}

// the reference's apply_green_kernel + normalisation, FP32, in place:
// -4 pi / k^2 * exp(-k^2 r_s^2) * 1/M^3; modes with max|k_i| < k_min and k = 0 zeroed
__global__ void k_kspace_rc(float2* __restrict__ data, int M, float dk, float rs2, float norm,
                            int k_min, int64_t Gc)
{
    int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= Gc) return;
    int Mh = M / 2 + 1;
    int kx = (int)(idx % Mh);
    int64_t r = idx / Mh;
    int ky = (int)(r % M);
    int kz = (int)(r / M);
    int ix = kx, iy = ky <= M / 2 ? ky : ky - M, iz = kz <= M / 2 ? kz : kz - M;
    int kmax = max(max(abs(ix), abs(iy)), abs(iz));
    float2 z = data[idx];
    float kxv = ix * dk, kyv = iy * dk, kzv = iz * dk;
    float k2 = kxv * kxv + kyv * kyv + kzv * kzv;
    if (kmax < k_min || k2 <= 0.0f) {
        data[idx] = make_float2(0.f, 0.f);
        return;
    }
    float green = -12.566370614f / k2 * expf(-k2 * rs2) * norm;
    data[idx] = make_float2(z.x * green, z.y * green);
}

}  // namespace

void jt_launch_deposit(const float4* pos0, int64_t n0, float q0, const float4* pos1, int64_t n1,
                       float q1, float* rho, int M, float L, int rcompat, cudaStream_t st)
{
    (void)rcompat;
    int64_t n = n0 + n1;
    if (n <= 0) return;
    k_deposit<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(pos0, n0, q0, pos1, n1, q1, rho, M,
                                                           0.5f * L, (float)M / L);
}

void jt_launch_rcompat_deposit(const float4* pos_caller, const int8_t* sign_caller, int64_t n_all,
                               const float mass[2], float* rho, int M, float box_half,
                               float inv_cell, float inv_vol, cudaStream_t st)
{
    if (n_all <= 0) return;
    k_deposit_rc<<<(unsigned)((n_all + 255) / 256), 256, 0, st>>>(
        pos_caller, sign_caller, n_all, mass[0], mass[1], rho, M, box_half, inv_cell, inv_vol);
}

// axis table: computed on the host in double, stored as float4 per index
void jt_launch_kspace(const cufftComplex* rho_k, cufftComplex* out, int M, double L, double r_s,
                      int k_min, int rcompat, cudaStream_t st)
{
    int64_t Gc = (int64_t)M * M * (M / 2 + 1);
    float norm = (float)(1.0 / ((double)M * M * M));
    unsigned g = (unsigned)((Gc + 255) / 256);
    if (rcompat) {
        k_kspace_rc<<<g, 256, 0, st>>>((float2*)out, M, (float)(2.0 * 3.14159265358979323846 / L),
                                       (float)(r_s * r_s), norm, k_min, Gc);
        return;
    }
    // the axis table lives right after the three spectra (allocated by the caller)
    const float4* axis = reinterpret_cast<const float4*>(out + 3 * Gc);
    k_kspace_acc<<<g, 256, 0, st>>>((const float2*)rho_k, (float2*)out, M, axis, norm, k_min, Gc);
}
