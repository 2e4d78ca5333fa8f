// The z transforms and the k-space multiply of a 512^3 PM grid in one kernel.
//
// A 3D real FFT is separable: the batch runs the two transforms over each
// (x, y) plane with cuFFT (a 2D R2C per plane: [z][ky][kx], kx = 0..M/2), then
// this kernel transforms each (kx, ky) column along z, forms the force
// spectra of the column (the k-space step of k_b_kspace: interlaced grids
// combined, Green's function with the assignment deconvolution, -i k_c), and
// transforms each of them back along z; cuFFT's 2D C2R per plane finishes the
// inverse.  Against three cuFFT passes per 3D transform plus a separate
// k-space kernel, the z passes of the 2 forward and 6 inverse transforms and
// the k-space traffic become one read of the two spectra and one write of
// the six: 32 NG Gc bytes.
//
// One CTA takes 8 consecutive kx of one ky (8 columns, 512 threads: 64 per
// column, the column index fastest, so that each warp's loads and stores are
// 4 rows of 64 contiguous bytes).  A 512-point transform is three radix-8
// stages over registers (each thread holds 8 values), with two exchanges
// through shared memory between them; the exchange layouts (row stride 72
// and 9, column stride 580 complex) keep every access at the 2-wavefront
// minimum of 8-byte loads.  Forward, n = t + 64 j, k = k1 + 8 k2 + 64 k3:
//   stage 1, thread t:        DFT8 over j,  times W512^(t k1)
//   stage 2, thread (k1, t2): DFT8 over j2 (t = t2 + 8 j2), times W64^(t2 k2)
//   stage 3, thread (k1, k2): DFT8 over t2 -> X[k1 + 8 k2 + 64 k3], k3 = 0..7
// and the inverse runs the stages backwards with conjugate twiddles
// (unnormalised, as cuFFT's).  Twiddles come from sincospif of exact
// arguments m / 256, stored as the matrices the stages read.
#include "jt_internal.cuh"

namespace {

constexpr int kM = 512, kMh = kM / 2 + 1;
constexpr int kC = 8;                           // columns per CTA
constexpr int kNT = kC * 64;                    // threads per CTA
constexpr int kCS = 580;                        // column stride of the exchange buffer (complex)
constexpr int kTilesX = (kMh + kC - 1) / kC;    // 33 column tiles per ky

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b)
{
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
// times -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ float2 mul_s(float2 a)
{
    return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// In-place 8-point DFT, e^{-2 pi i n k / 8} (INV: e^{+...}, unnormalised):
// three radix-2 levels.
template <bool INV>
__device__ __forceinline__ void dft8(float2 (&v)[8])
{
    const float r = 0.70710678118654752f;
    const float2 a0 = cadd(v[0], v[4]), a1 = csub(v[0], v[4]);
    const float2 a2 = cadd(v[2], v[6]), a3 = mul_s<INV>(csub(v[2], v[6]));
    const float2 a4 = cadd(v[1], v[5]), a5 = csub(v[1], v[5]);
    const float2 a6 = cadd(v[3], v[7]), a7 = mul_s<INV>(csub(v[3], v[7]));
    const float2 b0 = cadd(a0, a2), b2 = csub(a0, a2), b1 = cadd(a1, a3), b3 = csub(a1, a3);
    const float2 c0 = cadd(a4, a6), c2 = csub(a4, a6), c1 = cadd(a5, a7), c3 = csub(a5, a7);
    const float2 s2 = mul_s<INV>(c2);
    const float2 sc1 = mul_s<INV>(c1), sc3 = mul_s<INV>(c3);
    const float2 w1 = make_float2(r * (c1.x + sc1.x), r * (c1.y + sc1.y));   // e^{-+i pi/4} c1
    const float2 w3 = make_float2(r * (sc3.x - c3.x), r * (sc3.y - c3.y));   // e^{-+3i pi/4} c3
    v[0] = cadd(b0, c0);
    v[4] = csub(b0, c0);
    v[2] = cadd(b2, s2);
    v[6] = csub(b2, s2);
    v[1] = cadd(b1, w1);
    v[5] = csub(b1, w1);
    v[3] = cadd(b3, w3);
    v[7] = csub(b3, w3);
}

// Forward 512-point transform of one column (thread t = 0..63 of it):
// in v[j] = x[t + 64 j]; out v[k3] = X[k1 + 8 k2 + 64 k3], k1 = t >> 3,
// k2 = t & 7.  XA and XB are the column's two exchange buffers (576 complex
// each): every transform writes XA, then XB, so a buffer is rewritten only
// after the barrier that follows its last read, and two barriers per
// transform suffice.
__device__ __forceinline__ void fft512_fwd(float2 (&v)[8], float2* XA, float2* XB, const float2* tw1,
                                           const float2* tw2, int t)
{
    dft8<false>(v);
#pragma unroll
    for (int k1 = 1; k1 < 8; k1++) v[k1] = cmul(v[k1], tw1[k1 * 64 + t]);
#pragma unroll
    for (int k1 = 0; k1 < 8; k1++) XA[k1 * 72 + t] = v[k1];
    __syncthreads();
    {
        const int k1 = t >> 3, t2 = t & 7;
#pragma unroll
        for (int j2 = 0; j2 < 8; j2++) v[j2] = XA[k1 * 72 + t2 + 8 * j2];
        dft8<false>(v);
#pragma unroll
        for (int k2 = 1; k2 < 8; k2++) v[k2] = cmul(v[k2], tw2[k2 * 8 + t2]);
#pragma unroll
        for (int k2 = 0; k2 < 8; k2++) XB[(k1 * 8 + k2) * 9 + t2] = v[k2];
    }
    __syncthreads();
#pragma unroll
    for (int t2 = 0; t2 < 8; t2++) v[t2] = XB[t * 9 + t2];   // (k1 * 8 + k2) = t
    dft8<false>(v);
}

// Inverse of fft512_fwd (unnormalised): in v[k3] = X[k1 + 8 k2 + 64 k3];
// out v[j] = x[t + 64 j].  Same buffer order (XA, then XB).
__device__ __forceinline__ void fft512_inv(float2 (&v)[8], float2* XA, float2* XB, const float2* tw1,
                                           const float2* tw2, int t)
{
    dft8<true>(v);
    {
        const int k2 = t & 7;
#pragma unroll
        for (int t2 = 1; t2 < 8; t2++) v[t2] = cmulc(v[t2], tw2[t2 * 8 + k2]);
    }
#pragma unroll
    for (int t2 = 0; t2 < 8; t2++) XA[t * 9 + t2] = v[t2];
    __syncthreads();
    {
        const int k1 = t >> 3, t2 = t & 7;
#pragma unroll
        for (int k2 = 0; k2 < 8; k2++) v[k2] = XA[(k1 * 8 + k2) * 9 + t2];
        dft8<true>(v);
#pragma unroll
        for (int j2 = 0; j2 < 8; j2++) v[j2] = cmulc(v[j2], tw1[k1 * 64 + t2 + 8 * j2]);
#pragma unroll
        for (int j2 = 0; j2 < 8; j2++) XB[k1 * 72 + t2 + 8 * j2] = v[j2];
    }
    __syncthreads();
#pragma unroll
    for (int k1 = 0; k1 < 8; k1++) v[k1] = XB[k1 * 72 + t];
    dft8<true>(v);
}

// src 0: the signed source (B.rho_k -> B.force_k); src 1: the unsigned source
// of a screened box (B.rho_s_k -> B.force_s_k).  The k-space arithmetic is
// k_b_kspace's, element by element.
template <bool IL>
__global__ void __launch_bounds__(kNT, 2)
k_zfft_kspace(const jt_box_dev* __restrict__ boxes, const int64_t* __restrict__ zprefix, int nbox, int k_min,
              int src)
{
    extern __shared__ float2 zsm[];
    // twiddles as the two matrices the stages read, each indexed fastest by
    // the reading thread's own index (no bank conflicts):
    // tw1[k1 * 64 + t] = W512^(t k1), tw2[k2 * 8 + t2] = W64^(t2 k2) (symmetric)
    float2* tw1 = zsm;
    float2* tw2 = zsm + kM;
    float2* xbuf = zsm + kM + 64;     // two exchange buffers per column
    const int64_t q = blockIdx.x;
    const int b = jt_find(zprefix, nbox, q);
    const jt_box_dev& B = boxes[b];
    const float2* __restrict__ in = src ? B.rho_s_k : B.rho_k;
    float2* __restrict__ out = src ? B.force_s_k : B.force_k;
    if (!in) return;   // the unsigned source of an unscreened box (whole block)
    const int64_t local = q - zprefix[b];
    const int ky = (int)(local / kTilesX);
    const int kx0 = (int)(local % kTilesX) * kC;
    const int tid = threadIdx.x, col = tid & (kC - 1), t = tid >> 3;
    const int kx = kx0 + col;
    const bool colok = kx < kMh;
    {
        // W512^m = e^{-2 pi i m / 512}: sincospif of the exact argument m / 256
        float s, c;
        sincospif((float)(((tid & 63) * (tid >> 6)) & (kM - 1)) * (1.0f / 256.0f), &s, &c);
        tw1[tid] = make_float2(c, -s);
        if (tid < 64) {
            sincospif((float)((8 * (tid & 7) * (tid >> 3)) & (kM - 1)) * (1.0f / 256.0f), &s, &c);
            tw2[tid] = make_float2(c, -s);
        }
    }
    __syncthreads();
    float2* XA = xbuf + col * kCS;
    float2* XB = xbuf + (kC + col) * kCS;
    const int64_t Gc = (int64_t)kM * kM * kMh;
    const int64_t sz = (int64_t)kMh * kM;   // z stride of a column
    const int64_t cb = (int64_t)(colok ? kx : 0) + (int64_t)kMh * ky;
    float2 P[8], v[8];
#pragma unroll
    for (int j = 0; j < 8; j++) v[j] = colok ? __ldcs(in + cb + (t + 64 * j) * sz) : make_float2(0.f, 0.f);
    fft512_fwd(v, XA, XB, tw1, tw2, t);
#pragma unroll
    for (int k = 0; k < 8; k++) P[k] = v[k];
    if (IL) {
#pragma unroll
        for (int j = 0; j < 8; j++)
            v[j] = colok ? __ldcs(in + Gc + cb + (t + 64 * j) * sz) : make_float2(0.f, 0.f);
        fft512_fwd(v, XA, XB, tw1, tw2, t);
    }
    const float4* __restrict__ ta = B.tabs;
    const float4* __restrict__ tb = B.tabs + kM;
    const float4 ax = __ldg(&ta[colok ? kx : 0]), ay = __ldg(&ta[ky]);
    const float4 bx = __ldg(&tb[colok ? kx : 0]), by = __ldg(&tb[ky]);
    const float2 exy = make_float2(bx.x * by.x - bx.y * by.y, bx.x * by.y + bx.y * by.x);
    const int half = kM / 2;
    const int nx = (int)ax.w, ny = (int)ay.w;
    const float norm = 1.0f / ((float)kM * (float)kM * (float)kM);
    const bool scr = B.ky2 > 0.0f;
    const int kz0 = (t >> 3) + 8 * (t & 7);   // k1 + 8 k2; kz = kz0 + 64 k3
#pragma unroll
    for (int k3 = 0; k3 < 8; k3++) {
        const int kz = kz0 + 64 * k3;
        const float4 az = __ldg(&ta[kz]);
        const float k2 = ax.x * ax.x + ay.x * ay.x + az.x * az.x;
        const int nz = (int)az.w;
        const int kmax = max(max(nx, ny), nz);
        const bool keep = colok && k2 > 0.0f && kmax >= k_min && nx != half && ny != half && nz != half;
        float2 z = P[k3];
        if (IL) {
            const float4 bz = __ldg(&tb[kz]);
            const float er = exy.x * bz.x - exy.y * bz.y, ei = exy.x * bz.y + exy.y * bz.x;
            const float2 u = v[k3];
            z.x = 0.5f * (z.x + (u.x * er + u.y * ei));
            z.y = 0.5f * (z.y + (u.y * er - u.x * ei));
        }
        float green = -12.566370614f * norm * (ax.z * ay.z * az.z) / k2;
        if (scr) {
            const float gy = green * (k2 / (k2 + B.ky2)) * B.yfac;
            green = src ? 0.5f * (green - gy) : 0.5f * (green + gy);
        }
        P[k3] = keep ? make_float2(z.x * green, z.y * green) : make_float2(0.f, 0.f);
    }
    // the six force spectra (three components, times the interlaced grid's
    // phase for the second grid), each transformed back along z
#pragma unroll 1
    for (int s = 0; s < 3 * (IL ? 2 : 1); s++) {
        const int c = s % 3, g = s / 3;
#pragma unroll
        for (int k3 = 0; k3 < 8; k3++) {
            const int kz = kz0 + 64 * k3;
            const float d = c == 0 ? ax.y : (c == 1 ? ay.y : __ldg(&ta[kz]).y);
            float2 f = make_float2(d * P[k3].y, -d * P[k3].x);
            if (g == 1) {
                const float4 bz = __ldg(&tb[kz]);
                const float2 e = make_float2(exy.x * bz.x - exy.y * bz.y, exy.x * bz.y + exy.y * bz.x);
                f = cmul(f, e);
            }
            v[k3] = f;
        }
        fft512_inv(v, XA, XB, tw1, tw2, t);
        if (colok) {
            float2* o = out + (int64_t)s * Gc + cb;
#pragma unroll
            for (int j = 0; j < 8; j++) o[(t + 64 * j) * sz] = v[j];
        }
    }
}

}  // namespace

int jt_zfft_tiles(int M) { return M == kM ? kM * kTilesX : 0; }

int jt_b_zfft_kspace(const jt_box_dev* d_boxes, const int64_t* d_zprefix, int nbox, int64_t ntiles, int interlace,
                     int k_min, int src, cudaStream_t st)
{
    if (ntiles <= 0) return JT_OK;
    const unsigned g = (unsigned)ntiles;
    const int smem = (int)sizeof(float2) * (kM + 64 + 2 * kC * kCS);
    const void* f = interlace ? (const void*)k_zfft_kspace<true> : (const void*)k_zfft_kspace<false>;
    if (jt_smem_attr(f, smem) != JT_OK) return JT_ECUDA;
    if (interlace) k_zfft_kspace<true><<<g, kNT, smem, st>>>(d_boxes, d_zprefix, nbox, k_min, src);
    else k_zfft_kspace<false><<<g, kNT, smem, st>>>(d_boxes, d_zprefix, nbox, k_min, src);
    return JT_OK;
}
