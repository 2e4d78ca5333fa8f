// Morton keys and the onesweep LSD radix sort (sm_100a).
//
// Keys follow the reference's quantisation (src/nbody_gpu_twopass.rs:291-326,
// compute_morton_f32): scale = 1024 / (2 box_half) in float, (x + box_half) *
// scale, saturating float->unsigned conversion, clamp to 10 bits, bit i of each
// axis at bit 3i (+1 for y, +2 for z).  The reference sorts 64-bit keys
// (m30 << 32) | index with 8 passes of 8 bits (:1521-1658, :2400-2434); sorting
// (m30, index) pairs stably gives the same order, so the accurate mode sorts the
// 30-bit code alone (4 passes, ties keep the previous Morton order) and the
// compatibility path sorts (m30 << 32 | caller index) over only the digit
// positions that can be non-zero.
//
// Onesweep (one pass over the keys per digit): an upfront kernel histograms all
// digit positions at once; each sort pass is ONE kernel in which every tile of
// 4096 keys ranks its keys with warp-level multi-split (match.any), publishes
// its digit counts, and reads the exclusive prefix of the tiles before it by
// decoupled look-back.  Tiles take their index from an atomic counter, so a
// tile only ever waits for tiles that are already running; each wait is also
// bounded (JT_ERRBIT_LOOKBACK).  Keys are reordered in shared memory first so
// the global scatter writes runs of equal digits.
#include "jt_internal.cuh"

#include <algorithm>
#include <cstdio>

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096
constexpr int kSortWarps = kSortThreads / 32;
constexpr uint32_t kFlagAgg = 1u << 30;
constexpr uint32_t kFlagInc = 2u << 30;
constexpr uint32_t kValMask = (1u << 30) - 1;
constexpr int kLookbackLimit = 1 << 22;

struct Shifts { int s[8]; int n; };

__device__ __forceinline__ uint32_t spread10(uint32_t x)
{
    x &= 0x3FFu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

__global__ void k_morton(const float4* __restrict__ pos, const int* __restrict__ id,
                         int64_t n, float box_half, uint32_t* __restrict__ key32,
                         uint64_t* __restrict__ key64, uint32_t* __restrict__ vals)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 p = pos[i];
    float scale = 1024.0f / (2.0f * box_half);
    // (x + box_half) * scale without contraction, as the reference
    float x = __fmul_rn(__fadd_rn(p.x, box_half), scale);
    float y = __fmul_rn(__fadd_rn(p.y, box_half), scale);
    float z = __fmul_rn(__fadd_rn(p.z, box_half), scale);
    uint32_t ix = min(__float2uint_rz(x), 0x3FFu);
    uint32_t iy = min(__float2uint_rz(y), 0x3FFu);
    uint32_t iz = min(__float2uint_rz(z), 0x3FFu);
    uint32_t m = spread10(ix) | (spread10(iy) << 1) | (spread10(iz) << 2);
    if (key64) key64[i] = ((uint64_t)m << 32) | (uint32_t)id[i];
    else key32[i] = m;
    vals[i] = (uint32_t)i;
}

template <typename K>
__device__ __forceinline__ uint32_t digit_of(K k, int shift) { return (uint32_t)(k >> shift) & 0xFFu; }

template <typename K>
__global__ void __launch_bounds__(256) k_radix_hist(const K* __restrict__ keys, int64_t n,
                                                    Shifts sh, uint32_t* __restrict__ hist)
{
    __shared__ uint32_t s[8][256];
    for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) (&s[0][0])[i] = 0;
    __syncthreads();
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        K k = keys[i];
        for (int p = 0; p < sh.n; p++) atomicAdd(&s[p][digit_of(k, sh.s[p])], 1u);
    }
    __syncthreads();
    for (int p = 0; p < sh.n; p++) {
        uint32_t c = s[p][threadIdx.x];
        if (c) atomicAdd(&hist[p * 256 + threadIdx.x], c);
    }
}

// exclusive scan of each pass's 256 counts, in place (one block per pass)
__global__ void k_radix_scan(uint32_t* hist)
{
    __shared__ uint32_t wsum[8];
    uint32_t* h = hist + blockIdx.x * 256;
    int t = threadIdx.x, lane = t & 31, w = t >> 5;
    uint32_t v = h[t], x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    uint32_t add = 0;
    for (int i = 0; i < w; i++) add += wsum[i];
    h[t] = x - v + add;
}

__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p)
{
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(uint32_t* p, uint32_t v)
{
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Decoupled look-back for digit t from tile p down: adds the aggregates of
// earlier tiles until one publishes an inclusive prefix.  A status word that
// stays empty for `limit` polls makes it give up: it sets JT_ERRBIT_LOOKBACK
// (reported as JT_ETIMEDOUT) and returns what it has, so no wait is endless.
__device__ __forceinline__ uint32_t lookback(const uint32_t* status, int64_t p, int t, unsigned* err,
                                             int limit)
{
    uint32_t excl = 0;
    int spins = 0;
    for (;;) {
        uint32_t wv = ld_relaxed(status + p * 256 + t);
        uint32_t flag = wv & ~kValMask;
        if (flag == 0u) {
            if (++spins > limit) {
                atomicOr(err, JT_ERRBIT_LOOKBACK);
                break;
            }
            if (spins > 64) __nanosleep(32);
            continue;
        }
        excl += wv & kValMask;
        if (flag == kFlagInc || p == 0) break;
        --p;
    }
    return excl;
}

// The same bounded wait on a status row that nothing publishes (a test of
// the failure path: it must time out and report, and the context must stay
// usable).
__global__ void k_wait_probe(const uint32_t* status, unsigned* err, int limit)
{
    if (threadIdx.x < 32) (void)lookback(status, 0, threadIdx.x, err, limit);
}

template <typename K>
struct SortSmem {
    uint32_t whist[kSortWarps][256];
    uint32_t tile_start[256];
    uint32_t gofs[256];
    uint32_t wsum[kSortWarps];
    int tile;
    K keys[kSortTile];
    uint32_t vals[kSortTile];
};

template <typename K>
__global__ void __launch_bounds__(kSortThreads)
k_onesweep(const K* __restrict__ kin, K* __restrict__ kout, const uint32_t* __restrict__ vin,
           uint32_t* __restrict__ vout, int64_t n, int shift, const uint32_t* __restrict__ base,
           uint32_t* __restrict__ status, uint32_t* __restrict__ tile_ctr, unsigned* err)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SortSmem<K>& S = *reinterpret_cast<SortSmem<K>*>(smem_raw);
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    if (t == 0) S.tile = (int)atomicAdd(tile_ctr, 1u);
    for (int i = t; i < kSortWarps * 256; i += kSortThreads) (&S.whist[0][0])[i] = 0;
    __syncthreads();
    const int tile = S.tile;
    const int64_t seg = (int64_t)tile * kSortTile + warp * (32 * kSortItems);

    K k[kSortItems];
    uint32_t v[kSortItems], rank[kSortItems];
#pragma unroll
    for (int j = 0; j < kSortItems; j++) {
        int64_t idx = seg + j * 32 + lane;
        bool ok = idx < n;
        k[j] = ok ? kin[idx] : K(0);
        v[j] = ok ? vin[idx] : 0u;
    }
    const uint32_t lt_mask = (1u << lane) - 1u;
#pragma unroll
    for (int j = 0; j < kSortItems; j++) {
        bool ok = (seg + j * 32 + lane) < n;
        uint32_t d = digit_of(k[j], shift);
        uint32_t peers = __match_any_sync(0xffffffffu, ok ? d : (0x100u + lane));
        int leader = __ffs(peers) - 1;
        uint32_t old = 0;
        if (ok && lane == leader) {
            old = S.whist[warp][d];
            S.whist[warp][d] = old + __popc(peers);
        }
        old = __shfl_sync(0xffffffffu, old, leader);
        rank[j] = old + __popc(peers & lt_mask);
        __syncwarp();
    }
    __syncthreads();

    // per digit (thread t = digit): exclusive prefix over warps, tile count
    uint32_t count = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; w++) {
        uint32_t c = S.whist[w][t];
        S.whist[w][t] = count;
        count += c;
    }
    uint32_t* row = status + (int64_t)tile * 256;
    st_relaxed(row + t, (tile == 0 ? kFlagInc : kFlagAgg) | count);

    // tile-local digit starts: block exclusive scan of count
    uint32_t x = count;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) S.wsum[warp] = x;
    __syncthreads();
    uint32_t add = 0;
    for (int i = 0; i < warp; i++) add += S.wsum[i];
    S.tile_start[t] = x - count + add;

    // decoupled look-back for digit t
    uint32_t excl = 0;
    if (tile > 0) {
        excl = lookback(status, tile - 1, t, err, kLookbackLimit);
        st_relaxed(row + t, kFlagInc | (excl + count));
    }
    S.gofs[t] = base[t] + excl;
    __syncthreads();

    // stable local reorder by digit
#pragma unroll
    for (int j = 0; j < kSortItems; j++) {
        bool ok = (seg + j * 32 + lane) < n;
        if (ok) {
            uint32_t d = digit_of(k[j], shift);
            uint32_t pos = S.tile_start[d] + S.whist[warp][d] + rank[j];
            S.keys[pos] = k[j];
            S.vals[pos] = v[j];
        }
    }
    __syncthreads();
    int64_t rem = n - (int64_t)tile * kSortTile;
    int tile_n = rem < kSortTile ? (int)rem : kSortTile;
    for (int e = t; e < tile_n; e += kSortThreads) {
        K key = S.keys[e];
        uint32_t d = digit_of(key, shift);
        uint32_t dst = S.gofs[d] + (uint32_t)e - S.tile_start[d];
        kout[dst] = key;
        vout[dst] = S.vals[e];
    }
}

__global__ void k_reorder(const uint32_t* __restrict__ perm, int64_t n,
                          const float4* __restrict__ pin, float4* __restrict__ pout,
                          const float4* __restrict__ vin, float4* __restrict__ vout,
                          const int* __restrict__ iin, int* __restrict__ iout)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t s = perm[i];
    pout[i] = pin[s];
    if (vin) vout[i] = vin[s];
    iout[i] = iin[s];
}

__global__ void k_split_keys(const uint64_t* __restrict__ k, int64_t n, uint32_t* __restrict__ hi,
                             uint32_t* __restrict__ lo)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint64_t v = k[i];
    hi[i] = (uint32_t)(v >> 32);
    lo[i] = (uint32_t)v;
}

template <typename K>
int radix_sort(K* keys, uint32_t* vals, int64_t n, const int* shifts, int npass,
               jt_sort_ws* ws, unsigned* d_err, cudaStream_t st)
{
    if (n <= 1 || npass == 0) return 0;
    if (n > ws->cap || npass > ws->max_passes || npass > 8) return JT_EINVAL;
    if (n >= (int64_t)kValMask) return JT_EINVAL;
    Shifts sh;
    sh.n = npass;
    for (int p = 0; p < npass; p++) sh.s[p] = shifts[p];
    int64_t tiles = (n + kSortTile - 1) / kSortTile;
    cudaMemsetAsync(ws->hist, 0, sizeof(uint32_t) * 256 * npass, st);
    cudaMemsetAsync(ws->status, 0, sizeof(uint32_t) * 256 * tiles * npass, st);
    cudaMemsetAsync(ws->tile_ctr, 0, sizeof(uint32_t) * npass, st);
    int hb = (int)std::min<int64_t>((n + 255) / 256, 148 * 8);
    k_radix_hist<K><<<hb, 256, 0, st>>>(keys, n, sh, ws->hist);
    k_radix_scan<<<npass, 256, 0, st>>>(ws->hist);
    size_t smem = sizeof(SortSmem<K>);
    if (jt_smem_attr((const void*)k_onesweep<K>, (int)smem) != JT_OK) return JT_ECUDA;
    K* a = keys;
    K* b = reinterpret_cast<K*>(ws->keys_alt);
    uint32_t* va = vals;
    uint32_t* vb = ws->vals_alt;
    for (int p = 0; p < npass; p++) {
        k_onesweep<K><<<(unsigned)tiles, kSortThreads, smem, st>>>(
            a, b, va, vb, n, sh.s[p], ws->hist + p * 256, ws->status + (int64_t)p * tiles * 256,
            ws->tile_ctr + p, d_err);
        std::swap(a, b);
        std::swap(va, vb);
    }
    if (a != keys) {
        cudaMemcpyAsync(keys, a, sizeof(K) * n, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(vals, va, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : JT_ECUDA;
}

}  // namespace

int jt_sort_ws_alloc(jt_sort_ws* ws, int64_t cap, int max_passes)
{
    int64_t tiles = (cap + kSortTile - 1) / kSortTile;
    if (tiles < 1) tiles = 1;
    ws->cap = cap;
    ws->max_passes = max_passes;
    cudaError_t e = cudaSuccess;
    e = (e == cudaSuccess) ? cudaMalloc(&ws->keys_alt, sizeof(uint64_t) * (cap > 0 ? cap : 1)) : e;
    e = (e == cudaSuccess) ? cudaMalloc((void**)&ws->vals, sizeof(uint32_t) * (cap > 0 ? cap : 1)) : e;
    e = (e == cudaSuccess) ? cudaMalloc((void**)&ws->vals_alt, sizeof(uint32_t) * (cap > 0 ? cap : 1)) : e;
    e = (e == cudaSuccess) ? cudaMalloc((void**)&ws->hist, sizeof(uint32_t) * 256 * max_passes) : e;
    e = (e == cudaSuccess) ? cudaMalloc((void**)&ws->status, sizeof(uint32_t) * 256 * tiles * max_passes) : e;
    e = (e == cudaSuccess) ? cudaMalloc((void**)&ws->tile_ctr, sizeof(uint32_t) * max_passes) : e;
    return e == cudaSuccess ? 0 : JT_ENOMEM;
}

void jt_sort_ws_free(jt_sort_ws* ws)
{
    cudaFree(ws->keys_alt);
    cudaFree(ws->vals);
    cudaFree(ws->vals_alt);
    cudaFree(ws->hist);
    cudaFree(ws->status);
    cudaFree(ws->tile_ctr);
    *ws = jt_sort_ws{};
}

void jt_launch_morton(const float4* pos, const int* id, int64_t n, float box_half,
                      uint32_t* key32, uint64_t* key64, uint32_t* vals, cudaStream_t st)
{
    if (n <= 0) return;
    k_morton<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(pos, id, n, box_half, key32, key64, vals);
}

int jt_radix_sort_u64(uint64_t* keys, uint32_t* vals, int64_t n, const int* shifts, int npass,
                      jt_sort_ws* ws, unsigned* d_err, cudaStream_t st)
{
    return radix_sort<uint64_t>(keys, vals, n, shifts, npass, ws, d_err, st);
}

void jt_launch_reorder(const uint32_t* perm, int64_t n, const float4* pos_in, float4* pos_out,
                       const float4* vel_in, float4* vel_out, const int* id_in, int* id_out,
                       cudaStream_t st)
{
    if (n <= 0) return;
    k_reorder<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(perm, n, pos_in, pos_out, vel_in,
                                                           vel_out, id_in, id_out);
}

void jt_launch_split_keys(const uint64_t* key64, int64_t n, uint32_t* m30, uint32_t* tie,
                          cudaStream_t st)
{
    if (n <= 0) return;
    k_split_keys<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(key64, n, m30, tie);
}

// ======================================================================
// Batched (segmented) versions: one launch per stage for every segment
// (box x species) of a batch.  A segment's keys are its tree.m30 array.
// ======================================================================
namespace {

__global__ void k_b_morton(const jt_seg_dev* __restrict__ segs, const jt_box_dev* __restrict__ boxes,
                           const int64_t* __restrict__ prefix, int nseg)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= prefix[nseg]) return;
    const int g = jt_find(prefix, nseg, i);
    const int64_t j = i - prefix[g];
    const jt_seg_dev& S = segs[g];
    const float box_half = boxes[S.box].box_half;
    float4 p = S.pos[j];
    float scale = 1024.0f / (2.0f * box_half);
    float x = __fmul_rn(__fadd_rn(p.x, box_half), scale);
    float y = __fmul_rn(__fadd_rn(p.y, box_half), scale);
    float z = __fmul_rn(__fadd_rn(p.z, box_half), scale);
    uint32_t ix = min(__float2uint_rz(x), 0x3FFu);
    uint32_t iy = min(__float2uint_rz(y), 0x3FFu);
    uint32_t iz = min(__float2uint_rz(z), 0x3FFu);
    S.tree.m30[j] = spread10(ix) | (spread10(iy) << 1) | (spread10(iz) << 2);
    S.vals[j] = (uint32_t)j;
}

// per-segment histograms of the 4 digit positions (blocks over sort tiles)
__global__ void __launch_bounds__(256) k_b_hist(const jt_seg_dev* __restrict__ segs,
                                                const int64_t* __restrict__ tprefix, int nseg)
{
    __shared__ uint32_t s[4][256];
    const int64_t tile = blockIdx.x;
    const int g = jt_find(tprefix, nseg, tile);
    const jt_seg_dev& S = segs[g];
    const int64_t lt = tile - tprefix[g];
    for (int i = threadIdx.x; i < 4 * 256; i += blockDim.x) (&s[0][0])[i] = 0;
    __syncthreads();
    const int64_t b0 = lt * kSortTile, b1 = min((int64_t)S.n, b0 + kSortTile);
    for (int64_t i = b0 + threadIdx.x; i < b1; i += blockDim.x) {
        uint32_t k = S.tree.m30[i];
#pragma unroll
        for (int p = 0; p < 4; p++) atomicAdd(&s[p][(k >> (8 * p)) & 0xFFu], 1u);
    }
    __syncthreads();
#pragma unroll
    for (int p = 0; p < 4; p++) {
        uint32_t c = s[p][threadIdx.x];
        if (c) atomicAdd(&S.hist[p * 256 + threadIdx.x], c);
    }
}

// exclusive scan of each (segment, pass) histogram: block = 4 * segment + pass
__global__ void k_b_scan(const jt_seg_dev* __restrict__ segs)
{
    __shared__ uint32_t wsum[8];
    uint32_t* h = segs[blockIdx.x >> 2].hist + (blockIdx.x & 3) * 256;
    int t = threadIdx.x, lane = t & 31, w = t >> 5;
    uint32_t v = h[t], x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    uint32_t add = 0;
    for (int i = 0; i < w; i++) add += wsum[i];
    h[t] = x - v + add;
}

// One onesweep pass over every segment.  Tickets (atomic, global over the
// batch) are handed out in segment-then-tile order, so a tile only waits for
// tiles of its own segment that already hold lower tickets.  Even passes read
// (m30, vals) and write (keys_alt, vals_alt); odd passes the reverse.
// 4 blocks per SM (64 registers): the pass is latency-bound on its
// look-back, and the extra resident tiles hide more of it than the few
// spilled registers cost (1.62 -> 1.42 ms for the four passes at 2x224^3)
__global__ void __launch_bounds__(kSortThreads, 4)
k_b_onesweep(const jt_seg_dev* __restrict__ segs, const int64_t* __restrict__ tprefix, int nseg,
             int pass, uint32_t* __restrict__ ticket, unsigned* err)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    SortSmem<uint32_t>& S = *reinterpret_cast<SortSmem<uint32_t>*>(smem_raw);
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    if (t == 0) S.tile = (int)atomicAdd(ticket, 1u);
    for (int i = t; i < kSortWarps * 256; i += kSortThreads) (&S.whist[0][0])[i] = 0;
    __syncthreads();
    const int64_t gt = S.tile;
    const int g = jt_find(tprefix, nseg, gt);
    const jt_seg_dev& G = segs[g];
    const int tile = (int)(gt - tprefix[g]);
    const int64_t n = G.n;
    const int shift = 8 * pass;
    const uint32_t* kin = (pass & 1) ? G.keys_alt : G.tree.m30;
    uint32_t* kout = (pass & 1) ? G.tree.m30 : G.keys_alt;
    const uint32_t* vin = (pass & 1) ? G.vals_alt : G.vals;
    uint32_t* vout = (pass & 1) ? G.vals : G.vals_alt;
    const uint32_t* base = G.hist + pass * 256;
    const int64_t ntiles = (n + kSortTile - 1) / kSortTile;
    uint32_t* status = G.status + (int64_t)pass * ntiles * 256;
    const int64_t seg0 = (int64_t)tile * kSortTile + warp * (32 * kSortItems);

    uint32_t k[kSortItems], v[kSortItems], rank[kSortItems];
#pragma unroll
    for (int j = 0; j < kSortItems; j++) {
        int64_t idx = seg0 + j * 32 + lane;
        bool ok = idx < n;
        k[j] = ok ? kin[idx] : 0u;
        v[j] = ok ? vin[idx] : 0u;
    }
    const uint32_t lt_mask = (1u << lane) - 1u;
#pragma unroll
    for (int j = 0; j < kSortItems; j++) {
        bool ok = (seg0 + j * 32 + lane) < n;
        uint32_t d = (k[j] >> shift) & 0xFFu;
        uint32_t peers = __match_any_sync(0xffffffffu, ok ? d : (0x100u + lane));
        int leader = __ffs(peers) - 1;
        uint32_t old = 0;
        if (ok && lane == leader) {
            old = S.whist[warp][d];
            S.whist[warp][d] = old + __popc(peers);
        }
        old = __shfl_sync(0xffffffffu, old, leader);
        rank[j] = old + __popc(peers & lt_mask);
        __syncwarp();
    }
    __syncthreads();
    uint32_t count = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; w++) {
        uint32_t c = S.whist[w][t];
        S.whist[w][t] = count;
        count += c;
    }
    uint32_t* row = status + (int64_t)tile * 256;
    st_relaxed(row + t, (tile == 0 ? kFlagInc : kFlagAgg) | count);
    uint32_t x = count;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) S.wsum[warp] = x;
    __syncthreads();
    uint32_t add = 0;
    for (int i = 0; i < warp; i++) add += S.wsum[i];
    S.tile_start[t] = x - count + add;
    uint32_t excl = 0;
    if (tile > 0) {
        excl = lookback(status, tile - 1, t, err, kLookbackLimit);
        st_relaxed(row + t, kFlagInc | (excl + count));
    }
    S.gofs[t] = base[t] + excl;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kSortItems; j++) {
        bool ok = (seg0 + j * 32 + lane) < n;
        if (ok) {
            uint32_t d = (k[j] >> shift) & 0xFFu;
            uint32_t pos = S.tile_start[d] + S.whist[warp][d] + rank[j];
            S.keys[pos] = k[j];
            S.vals[pos] = v[j];
        }
    }
    __syncthreads();
    int64_t rem = n - (int64_t)tile * kSortTile;
    int tile_n = rem < kSortTile ? (int)rem : kSortTile;
    for (int e = t; e < tile_n; e += kSortThreads) {
        uint32_t key = S.keys[e];
        uint32_t d = (key >> shift) & 0xFFu;
        uint32_t dst = S.gofs[d] + (uint32_t)e - S.tile_start[d];
        kout[dst] = key;
        vout[dst] = S.vals[e];
    }
}

__global__ void k_b_reorder(const jt_seg_dev* __restrict__ segs, const int64_t* __restrict__ prefix,
                            int nseg)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= prefix[nseg]) return;
    const int g = jt_find(prefix, nseg, i);
    const int64_t j = i - prefix[g];
    const jt_seg_dev& S = segs[g];
    uint32_t s = S.vals[j];
    S.pos_b[j] = S.pos[s];
    S.vel_b[j] = S.vel[s];
    S.id_b[j] = S.id[s];
}

}  // namespace

// Sort every segment's particles by 30-bit Morton key (4 onesweep passes) and
// gather their state into the ping-pong buffers (the caller swaps them).
// pprefix: particles per segment; tprefix: sort tiles per segment (host and
// device copies); ws: per-pass ticket counters.
int jt_b_sort_reorder(const jt_seg_dev* d_segs, const jt_box_dev* d_boxes, int nseg,
                      const int64_t* d_pprefix, int64_t ntotal, const int64_t* d_tprefix,
                      int64_t ntiles, uint32_t* d_tickets, unsigned* d_err, cudaStream_t st)
{
    if (ntotal <= 0) return JT_OK;
    unsigned g = (unsigned)((ntotal + 255) / 256);
    k_b_morton<<<g, 256, 0, st>>>(d_segs, d_boxes, d_pprefix, nseg);
    k_b_hist<<<(unsigned)ntiles, 256, 0, st>>>(d_segs, d_tprefix, nseg);
    k_b_scan<<<4 * nseg, 256, 0, st>>>(d_segs);
    size_t smem = sizeof(SortSmem<uint32_t>);
    if (jt_smem_attr((const void*)k_b_onesweep, (int)smem) != JT_OK) return JT_ECUDA;
    for (int p = 0; p < 4; p++)
        k_b_onesweep<<<(unsigned)ntiles, kSortThreads, smem, st>>>(d_segs, d_tprefix, nseg, p,
                                                                   d_tickets + p, d_err);
    k_b_reorder<<<g, 256, 0, st>>>(d_segs, d_pprefix, nseg);
    return cudaGetLastError() == cudaSuccess ? JT_OK : JT_ECUDA;
}

int jt_sort_tile_size() { return kSortTile; }

extern "C" int jt_wait_probe(int limit, int* timed_out)
{
    if (limit <= 0 || limit > (1 << 24) || !timed_out) return JT_EINVAL;
    *timed_out = 0;
    uint32_t* status = nullptr;
    unsigned* err = nullptr;
    if (cudaMalloc(&status, 256 * sizeof(uint32_t)) != cudaSuccess) return JT_ENOMEM;
    if (cudaMalloc(&err, sizeof(unsigned)) != cudaSuccess) {
        cudaFree(status);
        return JT_ENOMEM;
    }
    int r = JT_OK;
    unsigned e = 0;
    if (cudaMemset(status, 0, 256 * sizeof(uint32_t)) != cudaSuccess || cudaMemset(err, 0, sizeof(unsigned)) != cudaSuccess)
        r = JT_ECUDA;
    if (r == JT_OK) {
        k_wait_probe<<<1, 32>>>(status, err, limit);
        if (cudaMemcpy(&e, err, sizeof(unsigned), cudaMemcpyDeviceToHost) != cudaSuccess) r = JT_ECUDA;
    }
    cudaFree(status);
    cudaFree(err);
    if (r != JT_OK) return r;
    *timed_out = (e & JT_ERRBIT_LOOKBACK) ? 1 : 0;
    return *timed_out ? JT_ETIMEDOUT : JT_OK;
}
