// Particle-mesh kernels: signed mass deposit and the fused k-space kernel.
//
// Reference: cic_scatter (src/nbody_gpu_twopass.rs:98-158) deposits counts of
// each species into two f64 grids with CAS-loop atomics; cufft_solve_device
// (cuda/cufft_wrapper.cu:350-398) then runs, per species, a D2D copy, D2Z,
// apply_green_kernel (:148-208), Z2D and a normalisation kernel, each followed
// by a device synchronisation.
//
// Here: one FP32 grid holds the signed source rho = sum_j s_j m_j W / h^3 of
// both species (the reference's F+ = -grad phi+ + grad phi- is the same linear
// combination).  Accurate mode:
//   * deposit: one CTA per Morton-aligned tile of T^3 cells.  Particles are
//     kept in Morton order, so a tile's particles are one contiguous range of
//     each species' array; the CTA accumulates them into a shared-memory copy
//     of the tile plus a halo with shared-memory fixed-point (int32) atomics
//     and flushes it to the grid with coalesced float4 global reductions.  CIC (8 cells)
//     or TSC (27 cells); with interlacing a second grid whose nodes sit half a
//     cell higher on every axis receives the same particles.
//   * one (batched) R2C; ONE k-space kernel combines the interlaced spectra,
//     applies -4 pi/k^2 x exp(-k^2 r_s^2) x 1/U(k)^2 (U = sinc^order per axis)
//     x 1/M^3, takes the spectral gradient -i k, and writes the three force
//     spectra (six with interlacing, the second three phase-shifted to the
//     shifted nodes); modes on a Nyquist plane are dropped (their weight is
//     exp(-(pi r_s/h)^2) ~ 2e-7 at r_s = 1.25 h); one batched C2R.
// Compatibility mode writes the potential spectrum only (the reference's
// Green, r_s = r_cut/3, k_min filter) and differentiates in real space as the
// reference does.
#include "jt_internal.cuh"

namespace {

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ uint32_t compact3(uint32_t x)
{
    x &= 0x09249249u;
    x = (x ^ (x >> 2)) & 0x030C30C3u;
    x = (x ^ (x >> 4)) & 0x0300F00Fu;
    x = (x ^ (x >> 8)) & 0x030000FFu;
    x = (x ^ (x >> 16)) & 0x000003FFu;
    return x;
}

__device__ __forceinline__ int64_t lower_bound_tile(const uint32_t* __restrict__ m30, int64_t n,
                                                    uint32_t key, int shift)
{
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        int64_t mid = (lo + hi) >> 1;
        if ((m30[mid] >> shift) < key) lo = mid + 1; else hi = mid;
    }
    return lo;
}

constexpr int kTileEdge = 16;

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

int jt_pm_tile_edge(int M) { return M < kTileEdge ? M : kTileEdge; }

void jt_launch_rcompat_deposit(const float4* pos_caller, const int8_t* sign_caller, int64_t n_all,
                               const float mass[2], float* rho, int M, float box_half,
                               float inv_cell, float inv_vol, cudaStream_t st)
{
    if (n_all <= 0) return;
    k_deposit_rc<<<(unsigned)((n_all + 255) / 256), 256, 0, st>>>(
        pos_caller, sign_caller, n_all, mass[0], mass[1], rho, M, box_half, inv_cell, inv_vol);
}

void jt_launch_kspace_rc(cufftComplex* data, int M, double L, double r_s, int k_min, cudaStream_t st)
{
    int64_t Gc = (int64_t)M * M * (M / 2 + 1);
    float norm = (float)(1.0 / ((double)M * M * M));
    unsigned g = (unsigned)((Gc + 255) / 256);
    k_kspace_rc<<<g, 256, 0, st>>>((float2*)data, M, (float)(2.0 * 3.14159265358979323846 / L),
                                   (float)(r_s * r_s), norm, k_min, Gc);
}

// ======================================================================
// Batched versions over boxes: one launch per stage for the whole batch.
// ======================================================================
namespace {

__global__ void k_b_tile_ranges(const jt_seg_dev* __restrict__ segs, const jt_box_dev* __restrict__ boxes,
                                const int64_t* __restrict__ tprefix, int nbox)
{
    int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= tprefix[nbox]) return;
    const int b = jt_find(tprefix, nbox, q);
    const jt_box_dev& B = boxes[b];
    const uint32_t t = (uint32_t)(q - tprefix[b]);
    int4 r = make_int4(0, 0, 0, 0);
    if (B.seg[0] >= 0) {
        const jt_seg_dev& S = segs[B.seg[0]];
        r.x = (int)lower_bound_tile(S.tree.m30, S.n, t, B.tile_shift);
        r.y = (int)lower_bound_tile(S.tree.m30, S.n, t + 1, B.tile_shift);
    }
    if (B.seg[1] >= 0) {
        const jt_seg_dev& S = segs[B.seg[1]];
        r.z = (int)lower_bound_tile(S.tree.m30, S.n, t, B.tile_shift);
        r.w = (int)lower_bound_tile(S.tree.m30, S.n, t + 1, B.tile_shift);
    }
    B.ranges[t] = r;
}

// Tiled deposit: one CTA per Morton-aligned tile of T^3 cells of one box.
// The tile's particles are one contiguous range of each species' sorted
// array (B.ranges); they are accumulated into a shared-memory copy of the
// tile plus a halo, then flushed to the grid with global reductions.  The
// halo holds every stencil of a particle inside the tile, the interlaced
// grid's half-cell shift included: S = T + 3 cells on y and z from the origin
// T t - 1 for CIC and TSC, S = T + 4 from T t - 2 for PCS; on x the rows start
// 4 cells below the tile (T t - 4, a multiple of
// 4) and are W = T + 8 cells wide, so that the flush reads and reduces four
// cells at a time (16-byte shared loads, one float4 global reduction per
// non-zero group; 16-byte aligned because M, the row start and the grid base
// are multiples of 4).  Stencils that leave the halo (a particle outside its
// tile after the drift) go straight to the grid with float atomics.
//
// Fixed point.  Shared-memory int32 atomicAdd runs at ~8 per clock per SM on
// B200, float atomicAdd at ~2.5 (measured), and the deposit issues 27 (TSC)
// per particle and grid.  So the tile accumulates integers in units u of the
// source: every partial sum of a cell is bounded by Q = wmax sum_tile |q|
// (wmax the stencil's largest weight product), and u = max(Q / 2^29,
// wmax max|q| / 2^22) keeps every sum below 2^30 and every contribution below
// 2^22, where x + 1.5 2^23 rounds it to the nearest integer in the float's
// bits (an FMA and an integer subtract per contribution, no float-to-int
// conversion).  Each contribution is rounded to u / 2 at most: relative to
// the tile's bound that is 2^-30 (2^-23 of one particle's full weight in a
// sparse tile), below the FP32 sums' own rounding of the densest cells.
// Integer sums do not depend on the order of the atomics, so a tile's
// values are reproducible.  TT: the tile edge as a constant (16, the edge of
// every grid of 16^3 and up) or 0 (read per box).
// 512 threads, 2 blocks per SM (the 69 KB tile allows 3 of 256): 32 warps
// per SM hide more of the shared-memory atomics' latency.
template <int ORDER, int NG, int TT>
__global__ void __launch_bounds__(512, 2)
k_b_deposit(const jt_seg_dev* __restrict__ segs, const jt_box_dev* __restrict__ boxes,
            const int64_t* __restrict__ tprefix, int nbox, int src)
{
    extern __shared__ int4 tile4[];
    int* tile = reinterpret_cast<int*>(tile4);
    const int64_t q = blockIdx.x;
    const int b = jt_find(tprefix, nbox, q);
    const jt_box_dev& B = boxes[b];
    if (src && !B.rho_s) return;   // the unsigned source of an unscreened box: not used
    const uint32_t t = (uint32_t)(q - tprefix[b]);
    const int T = TT > 0 ? TT : B.T, M = B.M;
    constexpr int kLo = ORDER == 4 ? 2 : 1;   // halo below the tile on y and z
    const int S = T + 2 + kLo, W = T + 8, W4 = W / 4;
    // plane pitch padded by 4 ints: with S W (a multiple of 32 at T = 16)
    // particles that differ only in z hit the same bank; the pad spreads
    // them (3.7 -> 2.8 wavefronts per atomic instruction on a Morton-ordered
    // lattice, simulated), and keeps planes 16-byte aligned
    const int SW = S * W + 4, SW4 = SW / 4;
    const int ax = (int)compact3(t) * T - 4;
    const int by = (int)compact3(t >> 1) * T - kLo;
    const int bz = (int)compact3(t >> 2) * T - kLo;
    const int4 r = B.ranges[t];
    const int n0 = r.y - r.x, n1 = r.w - r.z;
    if (n0 + n1 == 0) return;   // an empty tile adds nothing (whole block)
    const int nq = NG * S * S * W4;       // int4 words that hold nodes
    for (int c = threadIdx.x; c < NG * S * SW4; c += blockDim.x) tile4[c] = make_int4(0, 0, 0, 0);
    const int mask = M - 1;
    const int64_t G = (int64_t)M * M * M;
    const float halfL = B.halfL, hinv = B.h_inv;
    const float inv_vol = hinv * hinv * hinv;
    const float q0 = B.mass[0] * inv_vol, q1 = (src ? B.mass[1] : -B.mass[1]) * inv_vol;
    // the tile's fixed-point unit (see above)
    const float wmax = ORDER == 2 ? 1.0f : (ORDER == 3 ? 0.421875f : 0.2962963f);   // (3/4)^3, (2/3)^3
    const float qa0 = fabsf(q0), qa1 = fabsf(q1);
    const float bound = wmax * ((float)n0 * qa0 + (float)n1 * qa1);
    const float qmax = wmax * fmaxf(n0 ? qa0 : 0.0f, n1 ? qa1 : 0.0f);
    const float unit = fmaxf(bound * 0x1p-29f, qmax * 0x1p-22f);
    if (!(unit > 0.0f)) return;   // massless particles add nothing (whole block)
    const float inv_unit = 1.0f / unit;
    const float qs0 = q0 * inv_unit, qs1 = q1 * inv_unit;
    const float4* pos0 = B.seg[0] >= 0 ? segs[B.seg[0]].pos : nullptr;
    const float4* pos1 = B.seg[1] >= 0 ? segs[B.seg[1]].pos : nullptr;
    float* rho = src ? B.rho_s : B.rho;
    constexpr float kRound = 12582912.0f;   // 1.5 * 2^23: x + kRound holds round(x) in its low bits
    constexpr int kRoundBits = 0x4B400000;
    __syncthreads();
    // A crowded tile (a clump: many particles per cell) gives each thread a
    // run of consecutive particles, so that the lanes of a warp, whose
    // atomics meet in one instruction, sit far apart in the tile instead of
    // in the same few cells; integer sums do not depend on the order
    const int ntot = n0 + n1, tid = (int)threadIdx.x, nth = (int)blockDim.x;
    const int per = ntot > 2048 ? (ntot + nth - 1) / nth : 0;
    const int niter = per ? per : (ntot - tid + nth - 1) / nth;
    for (int i = 0; i < niter; i++) {
        const int k = per ? tid * per + i : tid + i * nth;
        if (k >= ntot) break;   // per > 0: the rest of this thread's run is past the end
        float4 p;
        float qq, qg;
        if (k < n0) { p = pos0[r.x + k]; qq = qs0; qg = q0; } else { p = pos1[r.z + k - n0]; qq = qs1; qg = q1; }
        float gx = (p.x + halfL) * hinv, gy = (p.y + halfL) * hinv, gz = (p.z + halfL) * hinv;
#pragma unroll
        for (int g = 0; g < NG; g++) {
            float sh = 0.5f * g;
            float wx[ORDER], wy[ORDER], wz[ORDER];
            int ix = jt_stencil<ORDER>(gx - sh, wx);
            int iy = jt_stencil<ORDER>(gy - sh, wy);
            int iz = jt_stencil<ORDER>(gz - sh, wz);
            int lx = ix - ax, ly = iy - by, lz = iz - bz;
            bool inside = lx >= 0 && ly >= 0 && lz >= 0 && lx + ORDER <= W && ly + ORDER <= S &&
                          lz + ORDER <= S;
            if (inside) {
                int* tb_ = tile + g * S * SW;
#pragma unroll
                for (int c = 0; c < ORDER; c++)
#pragma unroll
                    for (int bb = 0; bb < ORDER; bb++) {
                        float wyz = qq * wz[c] * wy[bb];
                        int* row = tb_ + (lz + c) * SW + (ly + bb) * W + lx;
#pragma unroll
                        for (int a = 0; a < ORDER; a++)
                            atomicAdd(row + a, __float_as_int(fmaf(wyz, wx[a], kRound)) - kRoundBits);
                    }
            } else {
                float* gb = rho + g * G;
#pragma unroll
                for (int c = 0; c < ORDER; c++)
#pragma unroll
                    for (int bb = 0; bb < ORDER; bb++) {
                        float wyz = qg * wz[c] * wy[bb];
                        int64_t row = ((int64_t)((iz + c) & mask) * M + ((iy + bb) & mask)) * M;
#pragma unroll
                        for (int a = 0; a < ORDER; a++) atomicAdd(gb + row + ((ix + a) & mask), wyz * wx[a]);
                    }
            }
        }
    }
    __syncthreads();
    for (int c = threadIdx.x; c < nq; c += blockDim.x) {
        const int qx = c % W4, row = c / W4;
        const int ly = row % S, gz = row / S;
        const int lz = gz % S, g = gz / S;
        const int4 v = tile4[gz * SW4 + ly * W4 + qx];
        if ((v.x | v.y | v.z | v.w) == 0) continue;
        const int64_t idx = ((int64_t)((bz + lz) & mask) * M + ((by + ly) & mask)) * M + ((ax + 4 * qx) & mask);
        atomicAdd(reinterpret_cast<float4*>(rho + g * G + idx),
                  make_float4((float)v.x * unit, (float)v.y * unit, (float)v.z * unit, (float)v.w * unit));
    }
}

// PM interpolation, tiled like the deposit: one CTA per (Morton tile of T^3
// cells of one box, interlaced grid b).  The three force grids of grid b
// over the tile plus its stencil halo, nodes T t - 2 .. T t + T + 1 on every
// axis (R = T + 4, the reach of CIC, TSC and PCS stencils of a particle in
// the tile, the interlaced grid's half-cell shift included), are staged in
// shared memory with asynchronous 8-byte copies (cp.async; R = 20 at
// T = 16: 96 KB, 2 blocks per SM).  The tile's particles (one contiguous
// range per species, B.ranges) are then interpolated by groups of 4 lanes:
// lane q of a group takes x offset q of all ORDER^2 stencil rows of every
// component (sums over y, then z, then one weight along x), so the 32 lanes
// of a load instruction read the rows of 8 particles, 4 consecutive floats
// each (few bank conflicts; one lane per particle reading its own 27-64
// scattered nodes conflicts ~4-way), and the group sums its partial forces
// with two shuffle steps.  Groups of 8 lanes (x offset and row parity)
// repeat the stencil arithmetic of a particle on twice the lanes: 5.06
// against 4.77 ms at 2x224^3; 16 lanes, one per (x, y) column, measured
// slower still (0.90 against 0.68 ms at 2x112^3).  A particle whose stencil leaves
// the region (outside its tile by the Morton key's rounding) reads the grid.
// Output: pmacc[b * npart + i] = the interpolated force of grid b on a unit
// m+ particle (i = the particle's index in the pass, pprefix[seg] + index);
// the walks average the grids and apply the sign.
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}

// 16-byte copy: both addresses 16-byte aligned
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

// TT: the tile edge as a constant (16, every grid of 16^3 and up: the
// region's index arithmetic folds) or 0 (read per box).  With TT = 16 a
// staged row of 20 nodes is stored rotated, [16 nodes of the tile | 2 above
// | 2 below], so that the tile's 16 nodes (64-byte aligned in the grid and
// in the row) travel as four 16-byte copies and each halo as one 8-byte
// copy: 6 copies per row instead of 10; node lx of the row sits at
// (lx + 18) % 20.
template <int ORDER, int TT>
__global__ void __launch_bounds__(512, 2)
k_b_interp(const jt_seg_dev* __restrict__ segs, const jt_box_dev* __restrict__ boxes,
           const int64_t* __restrict__ tprefix, const int64_t* __restrict__ pprefix, int nbox,
           int64_t npart, float4* __restrict__ pmacc)
{
    extern __shared__ float4 reg4[];
    float2* reg2 = reinterpret_cast<float2*>(reg4);
    const float* reg = reinterpret_cast<const float*>(reg4);
    const int64_t q = blockIdx.x;
    const int g = blockIdx.y;   // interlaced grid
    const int b = jt_find(tprefix, nbox, q);
    const jt_box_dev& B = boxes[b];
    if (g >= B.ngrid) return;
    const uint32_t t = (uint32_t)(q - tprefix[b]);
    const int4 r = B.ranges[t];
    const int n0 = r.y - r.x, n1 = r.w - r.z;
    if (n0 + n1 == 0) return;   // whole block
    const int T = TT > 0 ? TT : B.T, M = B.M, mask = M - 1, R = T + 4, RH = R / 2;
    const int ox = (int)compact3(t) * T - 2;
    const int oy = (int)compact3(t >> 1) * T - 2;
    const int oz = (int)compact3(t >> 2) * T - 2;
    const int64_t G = (int64_t)M * M * M;
    const float* __restrict__ F = B.force + (int64_t)g * 3 * G;
    const int rows = 3 * R * R;
    if (TT == 16) {
        float* regw = reinterpret_cast<float*>(reg4);
        for (int k = threadIdx.x; k < rows * 6; k += blockDim.x) {
            const int piece = k % 6, row = k / 6;
            const int y = row % R, zc = row / R;
            const int z = zc % R, c = zc / R;
            const int64_t rb = c * G + ((int64_t)((oz + z) & mask) * M + ((oy + y) & mask)) * M;
            float* dst = regw + row * R;
            if (piece < 4) cp_async16(dst + 4 * piece, F + rb + ox + 2 + 4 * piece);   // the tile's nodes
            else if (piece == 4) cp_async8(dst + 16, F + rb + ((ox + 18) & mask));     // 2 above
            else cp_async8(dst + 18, F + rb + (ox & mask));                            // 2 below
        }
    } else {
        // x pairs start at even nodes (ox and M even): 8-byte aligned, never split by the wrap
        for (int k = threadIdx.x; k < rows * RH; k += blockDim.x) {
            const int j = k % RH, row = k / RH;
            const int y = row % R, zc = row / R;
            const int z = zc % R, c = zc / R;
            const int64_t gi =
                c * G + ((int64_t)((oz + z) & mask) * M + ((oy + y) & mask)) * M + ((ox + 2 * j) & mask);
            cp_async8(reg2 + k, F + gi);
        }
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    const float halfL = B.halfL, hinv = B.h_inv, sh = 0.5f * g;
    const float4* pos0 = B.seg[0] >= 0 ? segs[B.seg[0]].pos : nullptr;
    const float4* pos1 = B.seg[1] >= 0 ? segs[B.seg[1]].pos : nullptr;
    const int64_t base0 = B.seg[0] >= 0 ? pprefix[B.seg[0]] : 0;
    const int64_t base1 = B.seg[1] >= 0 ? pprefix[B.seg[1]] : 0;
    float4* __restrict__ out = pmacc + (int64_t)g * npart;
    const int RR = R * R, RRR = RR * R;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const int gl = lane & 3;            // lane in the particle's group: x offset of the stencil
    const int n = n0 + n1;
    // every lane of a warp runs the same number of iterations (shuffles)
    for (int k0 = warp * 8; k0 < n; k0 += nwarp * 8) {
        const int k = k0 + (lane >> 2);
        const bool valid = k < n;
        float4 p = make_float4(0.f, 0.f, 0.f, 0.f);
        int64_t gi = 0;
        if (valid) {
            if (k < n0) { p = pos0[r.x + k]; gi = base0 + r.x + k; } else { p = pos1[r.z + k - n0]; gi = base1 + r.z + k - n0; }
        }
        float wx[ORDER], wy[ORDER], wz[ORDER];
        const int ix = jt_stencil<ORDER>((p.x + halfL) * hinv - sh, wx);
        const int iy = jt_stencil<ORDER>((p.y + halfL) * hinv - sh, wy);
        const int iz = jt_stencil<ORDER>((p.z + halfL) * hinv - sh, wz);
        const int lx = ix - ox, ly = iy - oy, lz = iz - oz;
        const bool in = lx >= 0 && ly >= 0 && lz >= 0 && lx + ORDER <= R && ly + ORDER <= R && lz + ORDER <= R;
        float ax = 0.f, ay = 0.f, az = 0.f;
        if (valid && gl < ORDER) {
            float wxq = wx[0];
#pragma unroll
            for (int a = 1; a < ORDER; a++) wxq = gl == a ? wx[a] : wxq;
            // the lane's column x = ix + gl of the stencil: sum over y, then z,
            // then one weight along x
            if (in) {
                const int xp = lx + gl;
                const float* base = reg + (lz * R + ly) * R + (TT == 16 ? (xp >= 2 ? xp - 2 : xp + 18) : xp);
#pragma unroll
                for (int zz = 0; zz < ORDER; zz++) {
                    float bx = 0.f, by = 0.f, bz = 0.f;
#pragma unroll
                    for (int yy = 0; yy < ORDER; yy++) {
                        const float* src = base + (zz * R + yy) * R;
                        bx = fmaf(wy[yy], src[0], bx);
                        by = fmaf(wy[yy], src[RRR], by);
                        bz = fmaf(wy[yy], src[2 * RRR], bz);
                    }
                    ax = fmaf(wz[zz], bx, ax);
                    ay = fmaf(wz[zz], by, ay);
                    az = fmaf(wz[zz], bz, az);
                }
            } else {
                const int64_t xg = (ix + gl) & mask;
#pragma unroll
                for (int zz = 0; zz < ORDER; zz++) {
                    float bx = 0.f, by = 0.f, bz = 0.f;
#pragma unroll
                    for (int yy = 0; yy < ORDER; yy++) {
                        const int64_t id = ((int64_t)((iz + zz) & mask) * M + ((iy + yy) & mask)) * M + xg;
                        bx = fmaf(wy[yy], __ldg(F + id), bx);
                        by = fmaf(wy[yy], __ldg(F + G + id), by);
                        bz = fmaf(wy[yy], __ldg(F + 2 * G + id), bz);
                    }
                    ax = fmaf(wz[zz], bx, ax);
                    ay = fmaf(wz[zz], by, ay);
                    az = fmaf(wz[zz], bz, az);
                }
            }
            ax *= wxq;
            ay *= wxq;
            az *= wxq;
        }
#pragma unroll
        for (int o = 1; o < 4; o <<= 1) {
            ax += __shfl_xor_sync(0xffffffffu, ax, o);
            ay += __shfl_xor_sync(0xffffffffu, ay, o);
            az += __shfl_xor_sync(0xffffffffu, az, o);
        }
        if (valid && gl == 0) out[gi] = make_float4(ax, ay, az, 0.f);
    }
}

// Fused k-space kernel, one thread per complex mode of one box.  Per-axis
// tables (index n = 0..M-1):
//   ta[n] = { k_n, gradient factor k_n (0 on the Nyquist plane),
//             exp(-k_n^2 r_s^2) / sinc^(2 order)(pi n/M), |n| }
//   tb[n] = { cos(k_n h/2), sin(k_n h/2), 0, 0 }   (interlacing phase)
// With interlacing rho = (rhoA + rhoB exp(-i theta)) / 2, theta = (kx+ky+kz) h/2,
// and the second set of force spectra is multiplied by exp(+i theta) so that
// its C2R gives the forces at the shifted nodes.  a_d(k) = -i k_d phi(k).
//
// A screened box (B.ky2 = kappa^2 > 0) also has the unsigned source S on
// rho_s_k.  With G_N the Green's function above and the Yukawa one
// G_Y = G_N k^2 / (k^2 + kappa^2) exp(-kappa^2 r_s^2) (the long part
// 4 pi exp(-(k^2 + kappa^2) r_s^2) / (k^2 + kappa^2) of e^{-kappa r} / r),
// D takes (G_N + G_Y) / 2 into force_k and S takes (G_N - G_Y) / 2 into
// force_s_k: a particle of sign s then feels s A_D + A_S, i.e. G_N from
// its own species and -G_Y from the other.
template <bool IL>
__global__ void k_b_kspace(const jt_box_dev* __restrict__ boxes, const int64_t* __restrict__ kprefix,
                           int nbox, int k_min)
{
    int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= kprefix[nbox]) return;
    const int b = jt_find(kprefix, nbox, q);
    const jt_box_dev& B = boxes[b];
    const int64_t idx = q - kprefix[b];
    const int M = B.M;
    const int64_t Gc = (int64_t)M * M * (M / 2 + 1);
    const float norm = 1.0f / ((float)M * (float)M * (float)M);
    const float4* ta = B.tabs;
    const float4* tb = B.tabs + M;
    const float2* rho_k = B.rho_k;
    float2* out = B.force_k;
    const int Mh = M / 2 + 1;
    const int kx = (int)(idx % Mh);
    const int64_t r = idx / Mh;
    const int ky = (int)(r % M);
    const int kz = (int)(r / M);
    const float4 ax = __ldg(&ta[kx]), ay = __ldg(&ta[ky]), az = __ldg(&ta[kz]);
    const float k2 = ax.x * ax.x + ay.x * ay.x + az.x * az.x;
    const int half = M / 2;
    const int nx = (int)ax.w, ny = (int)ay.w, nz = (int)az.w;
    const int kmax = max(max(nx, ny), nz);
    const bool keep = k2 > 0.0f && kmax >= k_min && nx != half && ny != half && nz != half;
    const bool scr = B.ky2 > 0.0f;
    float2 F0 = make_float2(0.f, 0.f), F1 = F0, F2 = F0, H0 = F0, H1 = F0, H2 = F0;
    float er = 1.0f, ei = 0.0f;
    if (keep) {
        float2 z = rho_k[idx];
        float2 zs = scr ? B.rho_s_k[idx] : make_float2(0.f, 0.f);
        if (IL) {
            float4 bx = __ldg(&tb[kx]), by = __ldg(&tb[ky]), bz = __ldg(&tb[kz]);
            float pr = bx.x * by.x - bx.y * by.y, pi = bx.x * by.y + bx.y * by.x;
            er = pr * bz.x - pi * bz.y;
            ei = pr * bz.y + pi * bz.x;
            float2 w = rho_k[Gc + idx];
            z.x = 0.5f * (z.x + (w.x * er + w.y * ei));
            z.y = 0.5f * (z.y + (w.y * er - w.x * ei));
            if (scr) {
                const float2 ws = B.rho_s_k[Gc + idx];
                zs.x = 0.5f * (zs.x + (ws.x * er + ws.y * ei));
                zs.y = 0.5f * (zs.y + (ws.y * er - ws.x * ei));
            }
        }
        float green = -12.566370614f * norm * (ax.z * ay.z * az.z) / k2;
        float gs = 0.0f;
        if (scr) {
            const float gy = green * (k2 / (k2 + B.ky2)) * B.yfac;
            gs = 0.5f * (green - gy);
            green = 0.5f * (green + gy);
        }
        float pr = z.x * green, pi = z.y * green;
        F0 = make_float2(ax.y * pi, -ax.y * pr);
        F1 = make_float2(ay.y * pi, -ay.y * pr);
        F2 = make_float2(az.y * pi, -az.y * pr);
        if (scr) {
            pr = zs.x * gs;
            pi = zs.y * gs;
            H0 = make_float2(ax.y * pi, -ax.y * pr);
            H1 = make_float2(ay.y * pi, -ay.y * pr);
            H2 = make_float2(az.y * pi, -az.y * pr);
        }
    }
    out[idx] = F0;
    out[Gc + idx] = F1;
    out[2 * Gc + idx] = F2;
    if (IL) {
        out[3 * Gc + idx] = make_float2(F0.x * er - F0.y * ei, F0.x * ei + F0.y * er);
        out[4 * Gc + idx] = make_float2(F1.x * er - F1.y * ei, F1.x * ei + F1.y * er);
        out[5 * Gc + idx] = make_float2(F2.x * er - F2.y * ei, F2.x * ei + F2.y * er);
    }
    if (scr) {
        float2* os = B.force_s_k;
        os[idx] = H0;
        os[Gc + idx] = H1;
        os[2 * Gc + idx] = H2;
        if (IL) {
            os[3 * Gc + idx] = make_float2(H0.x * er - H0.y * ei, H0.x * ei + H0.y * er);
            os[4 * Gc + idx] = make_float2(H1.x * er - H1.y * ei, H1.x * ei + H1.y * er);
            os[5 * Gc + idx] = make_float2(H2.x * er - H2.y * ei, H2.x * ei + H2.y * er);
        }
    }
}

}  // namespace

void jt_b_tile_ranges(const jt_seg_dev* d_segs, const jt_box_dev* d_boxes, const int64_t* d_tprefix,
                      int nbox, int64_t ntiles, cudaStream_t st)
{
    if (ntiles <= 0) return;
    k_b_tile_ranges<<<(unsigned)((ntiles + 255) / 256), 256, 0, st>>>(d_segs, d_boxes, d_tprefix, nbox);
}

// all boxes of a batch share order, ngrid and the tile edge T
int jt_b_deposit(const jt_seg_dev* d_segs, const jt_box_dev* d_boxes, const int64_t* d_tprefix,
                 int nbox, int64_t ntiles, int order, int ngrid, int T, cudaStream_t st, int src, bool T16)
{
    if (ntiles <= 0) return JT_OK;
    int S = T + (order == 4 ? 4 : 3), W = T + 8;
    size_t smem = sizeof(float) * (size_t)ngrid * S * (S * W + 4);   // padded plane pitch (k_b_deposit)
    // T16: every box of the pass has the tile edge 16 (T is the largest)
#define JT_BDEP1(O, NG, TT)                                                                   \
    do {                                                                                      \
        if (jt_smem_attr((const void*)k_b_deposit<O, NG, TT>, 96 * 1024) != JT_OK)            \
            return JT_ECUDA;                                                                  \
        k_b_deposit<O, NG, TT><<<(unsigned)ntiles, 512, smem, st>>>(d_segs, d_boxes, d_tprefix, nbox, src); \
    } while (0)
#define JT_BDEP(O, NG)                    \
    do {                                  \
        if (T16) JT_BDEP1(O, NG, 16);     \
        else JT_BDEP1(O, NG, 0);          \
    } while (0)
    if (order == 2 && ngrid == 1) JT_BDEP(2, 1);
    else if (order == 2 && ngrid == 2) JT_BDEP(2, 2);
    else if (order == 3 && ngrid == 1) JT_BDEP(3, 1);
    else if (order == 3 && ngrid == 2) JT_BDEP(3, 2);
    else if (order == 4 && ngrid == 1) JT_BDEP(4, 1);
    else if (order == 4 && ngrid == 2) JT_BDEP(4, 2);
    else return JT_EINVAL;
#undef JT_BDEP
#undef JT_BDEP1
    return cudaGetLastError() == cudaSuccess ? JT_OK : JT_ECUDA;
}

int jt_b_interp(const jt_seg_dev* d_segs, const jt_box_dev* d_boxes, const int64_t* d_tprefix,
                const int64_t* d_pprefix, int nbox, int64_t ntiles, int order, int ngrid, int T,
                int64_t npart, float4* pmacc, cudaStream_t st, bool T16)
{
    if (ntiles <= 0 || npart <= 0) return JT_OK;
    const int R = T + 4;
    const size_t smem = sizeof(float) * 3 * (size_t)R * R * R;
    if (smem > 200 * 1024) return JT_EINVAL;
    dim3 grid((unsigned)ntiles, (unsigned)ngrid);
#define JT_INTERP1(O, TT)                                                                              \
    do {                                                                                              \
        if (jt_smem_attr((const void*)k_b_interp<O, TT>, (int)smem) != JT_OK) return JT_ECUDA;        \
        k_b_interp<O, TT><<<grid, 512, smem, st>>>(d_segs, d_boxes, d_tprefix, d_pprefix, nbox, npart, pmacc); \
    } while (0)
#define JT_INTERP(O)                      \
    do {                                  \
        if (T16) JT_INTERP1(O, 16);       \
        else JT_INTERP1(O, 0);            \
    } while (0)
    if (order == 2) JT_INTERP(2);
    else if (order == 3) JT_INTERP(3);
    else if (order == 4) JT_INTERP(4);
    else return JT_EINVAL;
#undef JT_INTERP
#undef JT_INTERP1
    return cudaGetLastError() == cudaSuccess ? JT_OK : JT_ECUDA;
}

void jt_b_kspace(const jt_box_dev* d_boxes, const int64_t* d_kprefix, int nbox, int64_t nmodes,
                 int interlace, int k_min, cudaStream_t st)
{
    if (nmodes <= 0) return;
    unsigned g = (unsigned)((nmodes + 255) / 256);
    if (interlace) k_b_kspace<true><<<g, 256, 0, st>>>(d_boxes, d_kprefix, nbox, k_min);
    else k_b_kspace<false><<<g, 256, 0, st>>>(d_boxes, d_kprefix, nbox, k_min);
}
