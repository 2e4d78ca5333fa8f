// The z transforms and the k-space multiply of a 512^3 or 256^3 PM grid in
// one kernel.
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
// At 512^3 one CTA takes 8 consecutive kx of one ky (512 threads: 64 per
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
// (unnormalised, as cuFFT's).  At 256^3 (fft256_fwd below) a CTA takes 16
// columns of 32 threads and the last stage is two radix-4 DFTs per thread.
// Twiddles come from sincospif of exact arguments 2 m / M, stored as the
// matrices the stages read.
#include "jt_internal.cuh"

namespace {

constexpr int kNT = 512;   // threads per CTA (8 columns x 64 at 512^3, 16 x 32 at 256^3)

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

// w^1 .. w^7 from w (products at most three deep: about 3 ulp), in place of
// seven table loads (the shared-memory queue is the kernel's limit)
__device__ __forceinline__ void powers7(float2 w, float2 (&p)[8])
{
    p[1] = w;
    p[2] = cmul(w, w);
    p[3] = cmul(p[2], w);
    p[4] = cmul(p[2], p[2]);
    p[5] = cmul(p[4], w);
    p[6] = cmul(p[4], p[2]);
    p[7] = cmul(p[4], p[3]);
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
    {
        float2 w[8];
        powers7(tw1[64 + t], w);   // W512^(t k1), k1 = 1..7
#pragma unroll
        for (int k1 = 1; k1 < 8; k1++) v[k1] = cmul(v[k1], w[k1]);
    }
#pragma unroll
    for (int k1 = 0; k1 < 8; k1++) XA[k1 * 72 + t] = v[k1];
    __syncthreads();
    {
        const int k1 = t >> 3, t2 = t & 7;
#pragma unroll
        for (int j2 = 0; j2 < 8; j2++) v[j2] = XA[k1 * 72 + t2 + 8 * j2];
        dft8<false>(v);
        float2 w[8];
        powers7(tw2[8 + t2], w);   // W64^(t2 k2), k2 = 1..7
#pragma unroll
        for (int k2 = 1; k2 < 8; k2++) v[k2] = cmul(v[k2], w[k2]);
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
        float2 w[8];
        powers7(tw2[8 + (t & 7)], w);   // W64^(t2 k2), t2 = 1..7, k2 = t & 7
#pragma unroll
        for (int t2 = 1; t2 < 8; t2++) v[t2] = cmulc(v[t2], w[t2]);
    }
#pragma unroll
    for (int t2 = 0; t2 < 8; t2++) XA[t * 9 + t2] = v[t2];
    __syncthreads();
    {
        const int k1 = t >> 3, t2 = t & 7;
#pragma unroll
        for (int k2 = 0; k2 < 8; k2++) v[k2] = XA[(k1 * 8 + k2) * 9 + t2];
        dft8<true>(v);
        {
            // W512^((t2 + 8 j2) k1) = W512^(t2 k1) (W64^k1)^j2
            const float2 b = tw1[k1 * 64 + t2];
            float2 s[8];
            powers7(tw1[k1 * 64 + 8], s);
            v[0] = cmulc(v[0], b);
#pragma unroll
            for (int j2 = 1; j2 < 8; j2++) v[j2] = cmulc(v[j2], cmul(b, s[j2]));
        }
#pragma unroll
        for (int j2 = 0; j2 < 8; j2++) XB[k1 * 72 + t2 + 8 * j2] = v[j2];
    }
    __syncthreads();
#pragma unroll
    for (int k1 = 0; k1 < 8; k1++) v[k1] = XB[k1 * 72 + t];
    dft8<true>(v);
}

// In-place 4-point DFT (INV: e^{+...}, unnormalised).
template <bool INV>
__device__ __forceinline__ void dft4(float2& a0, float2& a1, float2& a2, float2& a3)
{
    const float2 b0 = cadd(a0, a2), b1 = csub(a0, a2), b2 = cadd(a1, a3), b3 = mul_s<INV>(csub(a1, a3));
    a0 = cadd(b0, b2);
    a2 = csub(b0, b2);
    a1 = cadd(b1, b3);
    a3 = csub(b1, b3);
}

// The 256-point transform of 256^3 grids: 32 threads per column, each holding
// 8 values; 256 = 8 x 8 x 4, n = t + 32 j, k = k1 + 8 k2 + 64 k3:
//   stage 1, thread t:        DFT8 over j,  times W256^(t k1)
//   stage 2, thread (k1, t2): DFT8 over j2 (t = t2 + 4 j2), times W32^(t2 k2)
//   stage 3, thread u takes the pairs p = u and u + 32 (k1 = p >> 3,
//            k2 = p & 7): DFT4 over t2 -> X[k1 + 8 k2 + 64 k3], k3 = 0..3,
//            held as v[4 h + k3] for p = u + 32 h
// Exchange layouts: row strides 32 and 4, column stride 257 (16 columns per
// CTA, the column index fastest in a warp: rows of 128 bytes); twiddle
// matrices tw1[k1 * 32 + t] = W256^(t k1), tw2[k2 * 4 + t2] = W32^(t2 k2).
__device__ __forceinline__ void fft256_fwd(float2 (&v)[8], float2* XA, float2* XB, const float2* tw1,
                                           const float2* tw2, int u)
{
    dft8<false>(v);
    {
        float2 w[8];
        powers7(tw1[32 + u], w);   // W256^(u k1), k1 = 1..7
#pragma unroll
        for (int k1 = 1; k1 < 8; k1++) v[k1] = cmul(v[k1], w[k1]);
    }
#pragma unroll
    for (int k1 = 0; k1 < 8; k1++) XA[k1 * 32 + u] = v[k1];
    __syncthreads();
    {
        const int k1 = u >> 2, t2 = u & 3;
#pragma unroll
        for (int j2 = 0; j2 < 8; j2++) v[j2] = XA[k1 * 32 + t2 + 4 * j2];
        dft8<false>(v);
        float2 w[8];
        powers7(tw2[4 + t2], w);   // W32^(t2 k2), k2 = 1..7
#pragma unroll
        for (int k2 = 1; k2 < 8; k2++) v[k2] = cmul(v[k2], w[k2]);
#pragma unroll
        for (int k2 = 0; k2 < 8; k2++) XB[(k1 * 8 + k2) * 4 + t2] = v[k2];
    }
    __syncthreads();
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int p = u + 32 * h;
#pragma unroll
        for (int t2 = 0; t2 < 4; t2++) v[4 * h + t2] = XB[p * 4 + t2];
        dft4<false>(v[4 * h], v[4 * h + 1], v[4 * h + 2], v[4 * h + 3]);
    }
}

// Inverse of fft256_fwd (unnormalised): in v[4 h + k3]; out v[j] = x[u + 32 j].
__device__ __forceinline__ void fft256_inv(float2 (&v)[8], float2* XA, float2* XB, const float2* tw1,
                                           const float2* tw2, int u)
{
    const int k2p = u & 7;   // k2 of both pairs (p = u, u + 32)
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int p = u + 32 * h;
        dft4<true>(v[4 * h], v[4 * h + 1], v[4 * h + 2], v[4 * h + 3]);
#pragma unroll
        for (int t2 = 0; t2 < 4; t2++) {
            const float2 c = t2 ? cmulc(v[4 * h + t2], tw2[k2p * 4 + t2]) : v[4 * h];
            XA[p * 4 + t2] = c;
        }
    }
    __syncthreads();
    {
        const int k1 = u >> 2, t2 = u & 3;
#pragma unroll
        for (int k2 = 0; k2 < 8; k2++) v[k2] = XA[(k1 * 8 + k2) * 4 + t2];
        dft8<true>(v);
        {
            // W256^((t2 + 4 j2) k1) = W256^(t2 k1) (W64^k1)^j2
            const float2 b = tw1[k1 * 32 + t2];
            float2 s[8];
            powers7(tw1[k1 * 32 + 4], s);
            v[0] = cmulc(v[0], b);
#pragma unroll
            for (int j2 = 1; j2 < 8; j2++) v[j2] = cmulc(v[j2], cmul(b, s[j2]));
        }
#pragma unroll
        for (int j2 = 0; j2 < 8; j2++) XB[k1 * 32 + t2 + 4 * j2] = v[j2];
    }
    __syncthreads();
#pragma unroll
    for (int k1 = 0; k1 < 8; k1++) v[k1] = XB[k1 * 32 + u];
    dft8<true>(v);
}

// Per grid size: columns per CTA, threads per column, exchange-buffer column
// stride (complex), twiddle entries (tw1 then tw2).
template <int M> struct ZShape;
template <> struct ZShape<512> {
    static constexpr int C = 8, T = 64, CS = 580, NTW1 = 512, NTW2 = 64;
};
template <> struct ZShape<256> {
    static constexpr int C = 16, T = 32, CS = 257, NTW1 = 256, NTW2 = 32;
};

template <int M> __host__ __device__ constexpr int z_tiles_x() { return (M / 2 + 1 + ZShape<M>::C - 1) / ZShape<M>::C; }

// the z frequency of the value v[i] that thread t holds after a forward transform
template <int M>
__device__ __forceinline__ int kz_of(int t, int i)
{
    if (M == 512) return (t >> 3) + 8 * (t & 7) + 64 * i;
    const int p = t + 32 * (i >> 2);
    return (p >> 3) + 8 * (p & 7) + 64 * (i & 3);
}

// One CTA of one box: 8 (512^3) or 16 (256^3) consecutive kx of one ky.
// src 0: the signed source (B.rho_k -> B.force_k); src 1: the unsigned source
// of a screened box (B.rho_s_k -> B.force_s_k).  The k-space arithmetic is
// k_b_kspace's, element by element.
template <int M, bool IL>
__device__ __forceinline__ void zfft_body(const jt_box_dev& B, const float2* __restrict__ in,
                                          float2* __restrict__ out, int64_t local, int k_min, int src,
                                          float2* zsm)
{
    using S = ZShape<M>;
    constexpr int Mh = M / 2 + 1, C = S::C, T = S::T, CS = S::CS;
    // twiddles as the two matrices the stages read, each indexed fastest by
    // the reading thread's own index (no bank conflicts)
    float2* tw1 = zsm;
    float2* tw2 = zsm + S::NTW1;
    float2* xbuf = zsm + S::NTW1 + S::NTW2;   // two exchange buffers per column
    const int ky = (int)(local / z_tiles_x<M>());
    const int kx0 = (int)(local % z_tiles_x<M>()) * C;
    const int tid = threadIdx.x, col = tid & (C - 1), t = tid / C;
    const int kx = kx0 + col;
    const bool colok = kx < Mh;
    {
        // W_M^m = e^{-2 pi i m / M}: sincospif of the exact argument 2 m / M
        float s, c;
        if (tid < S::NTW1) {
            const int k1 = tid / T, tt = tid % T;
            sincospif((float)((tt * k1) & (M - 1)) * (2.0f / M), &s, &c);
            tw1[tid] = make_float2(c, -s);
        }
        if (tid < S::NTW2) {
            // W(8 T)^(t2 k2) = W_M^(8 t2 k2): tw2[k2 * (T / 8) + t2]
            const int k2 = tid / (T / 8), t2 = tid % (T / 8);
            sincospif((float)((8 * t2 * k2) & (M - 1)) * (2.0f / M), &s, &c);
            tw2[tid] = make_float2(c, -s);
        }
    }
    __syncthreads();
    float2* XA = xbuf + col * CS;
    float2* XB = xbuf + (C + col) * CS;
    const int64_t Gc = (int64_t)M * M * Mh;
    const int64_t sz = (int64_t)Mh * M;   // z stride of a column
    const int64_t cb = (int64_t)(colok ? kx : 0) + (int64_t)Mh * ky;
    float2 P[8], v[8];
#pragma unroll
    for (int j = 0; j < 8; j++) v[j] = colok ? __ldcs(in + cb + (t + T * j) * sz) : make_float2(0.f, 0.f);
    if constexpr (M == 512) fft512_fwd(v, XA, XB, tw1, tw2, t);
    else fft256_fwd(v, XA, XB, tw1, tw2, t);
#pragma unroll
    for (int k = 0; k < 8; k++) P[k] = v[k];
    if (IL) {
#pragma unroll
        for (int j = 0; j < 8; j++)
            v[j] = colok ? __ldcs(in + Gc + cb + (t + T * j) * sz) : make_float2(0.f, 0.f);
        if constexpr (M == 512) fft512_fwd(v, XA, XB, tw1, tw2, t);
        else fft256_fwd(v, XA, XB, tw1, tw2, t);
    }
    const float4* __restrict__ ta = B.tabs;
    const float4* __restrict__ tb = B.tabs + M;
    const float4 ax = __ldg(&ta[colok ? kx : 0]), ay = __ldg(&ta[ky]);
    const float4 bx = __ldg(&tb[colok ? kx : 0]), by = __ldg(&tb[ky]);
    const float2 exy = make_float2(bx.x * by.x - bx.y * by.y, bx.x * by.y + bx.y * by.x);
    const int half = M / 2;
    const int nx = (int)ax.w, ny = (int)ay.w;
    const float norm = 1.0f / ((float)M * (float)M * (float)M);
    const bool scr = B.ky2 > 0.0f;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int kz = kz_of<M>(t, i);
        const float4 az = __ldg(&ta[kz]);
        const float k2 = ax.x * ax.x + ay.x * ay.x + az.x * az.x;
        const int nz = (int)az.w;
        const int kmax = max(max(nx, ny), nz);
        const bool keep = colok && k2 > 0.0f && kmax >= k_min && nx != half && ny != half && nz != half;
        float2 z = P[i];
        if (IL) {
            const float4 bz = __ldg(&tb[kz]);
            const float er = exy.x * bz.x - exy.y * bz.y, ei = exy.x * bz.y + exy.y * bz.x;
            const float2 u = v[i];
            z.x = 0.5f * (z.x + (u.x * er + u.y * ei));
            z.y = 0.5f * (z.y + (u.y * er - u.x * ei));
        }
        float green = -12.566370614f * norm * (ax.z * ay.z * az.z) / k2;
        if (scr) {
            const float gy = green * (k2 / (k2 + B.ky2)) * B.yfac;
            green = src ? 0.5f * (green - gy) : 0.5f * (green + gy);
        }
        P[i] = keep ? make_float2(z.x * green, z.y * green) : make_float2(0.f, 0.f);
    }
    // the six force spectra (three components, times the interlaced grid's
    // phase for the second grid), each transformed back along z
#pragma unroll 1
    for (int s = 0; s < 3 * (IL ? 2 : 1); s++) {
        const int c = s % 3, g = s / 3;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const int kz = kz_of<M>(t, i);
            const float dd = c == 0 ? ax.y : (c == 1 ? ay.y : __ldg(&ta[kz]).y);
            float2 f = make_float2(dd * P[i].y, -dd * P[i].x);
            if (g == 1) {
                const float4 bz = __ldg(&tb[kz]);
                const float2 e = make_float2(exy.x * bz.x - exy.y * bz.y, exy.x * bz.y + exy.y * bz.x);
                f = cmul(f, e);
            }
            v[i] = f;
        }
        if constexpr (M == 512) fft512_inv(v, XA, XB, tw1, tw2, t);
        else fft256_inv(v, XA, XB, tw1, tw2, t);
        if (colok) {
            float2* o = out + (int64_t)s * Gc + cb;
#pragma unroll
            for (int j = 0; j < 8; j++) o[(t + T * j) * sz] = v[j];
        }
    }
}

// One launch per grid size present in the pass (each with its own register
// allocation); the CTAs of the other size's boxes return at once.
template <int M, bool IL>
__global__ void __launch_bounds__(kNT, 2)
k_zfft_kspace(const jt_box_dev* __restrict__ boxes, const int64_t* __restrict__ zprefix, int nbox, int k_min,
              int src)
{
    extern __shared__ float2 zsm[];
    const int64_t q = blockIdx.x;
    const int b = jt_find(zprefix, nbox, q);
    const jt_box_dev& B = boxes[b];
    if (B.M != M) return;   // whole block
    const float2* __restrict__ in = src ? B.rho_s_k : B.rho_k;
    float2* __restrict__ out = src ? B.force_s_k : B.force_k;
    if (!in) return;   // the unsigned source of an unscreened box (whole block)
    zfft_body<M, IL>(B, in, out, q - zprefix[b], k_min, src, zsm);
}

}  // namespace

int jt_zfft_tiles(int M)
{
    if (M == 512) return 512 * z_tiles_x<512>();
    if (M == 256) return 256 * z_tiles_x<256>();
    return 0;
}

int jt_b_zfft_kspace(const jt_box_dev* d_boxes, const int64_t* d_zprefix, int nbox, int64_t ntiles, int interlace,
                     int k_min, int src, int sizes, cudaStream_t st)
{
    if (ntiles <= 0) return JT_OK;
    const unsigned g = (unsigned)ntiles;
#define JT_ZLAUNCH(MM)                                                                                   \
    do {                                                                                                 \
        const int smem = (int)sizeof(float2) *                                                           \
                         (ZShape<MM>::NTW1 + ZShape<MM>::NTW2 + 2 * ZShape<MM>::C * ZShape<MM>::CS);     \
        const void* f = interlace ? (const void*)k_zfft_kspace<MM, true> : (const void*)k_zfft_kspace<MM, false>; \
        if (jt_smem_attr(f, smem) != JT_OK) return JT_ECUDA;                                             \
        if (interlace) k_zfft_kspace<MM, true><<<g, kNT, smem, st>>>(d_boxes, d_zprefix, nbox, k_min, src);   \
        else k_zfft_kspace<MM, false><<<g, kNT, smem, st>>>(d_boxes, d_zprefix, nbox, k_min, src);          \
    } while (0)
    if (sizes & 1) JT_ZLAUNCH(512);
    if (sizes & 2) JT_ZLAUNCH(256);
#undef JT_ZLAUNCH
    return JT_OK;
}
