// Allocation-free variant of the Morton-key sort (jt_morton_sort_static).
//
// The sort behind jt_debug_tree (Morton keys -> onesweep LSD radix sort of
// (m30 << 32 | index) -> split into sorted codes and permutation) needs
// scratch: a key ping-pong buffer, two value buffers, digit histograms and
// the per-tile look-back words.  Here all of it lives in ONE file-scope
// static device array of fixed size, so the entry point calls no allocator:
// no cudaMalloc/cudaFree and no library call that allocates.  Its address is
// looked up once per device (cudaGetSymbolAddress with that device current)
// and cached.
//
// Layout of the array for n <= kMax elements (every region 256-byte aligned):
//   key64 [kMax] u64 | keys_alt [kMax] u64 | vals [kMax] u32 | vals_alt [kMax] u32
//   | hist [8][256] u32 | status [8][kMaxTiles][256] u32 | tile_ctr [8] u32
//   | err u32
// The array keeps the last call's contents; two calls that overlap in time
// race on it.
#include "jt_internal.cuh"

#include <mutex>

namespace {

constexpr int64_t kMax = JT_STATIC_SORT_MAX;
constexpr int64_t kTile = 4096;                        // onesweep tile (jt_sort.cu)
constexpr int64_t kMaxTiles = (kMax + kTile - 1) / kTile;
constexpr int kMaxPasses = 8;

constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kOffKey = 0;
constexpr size_t kOffKeyAlt = align256(kOffKey + 8 * kMax);
constexpr size_t kOffVals = align256(kOffKeyAlt + 8 * kMax);
constexpr size_t kOffValsAlt = align256(kOffVals + 4 * kMax);
constexpr size_t kOffHist = align256(kOffValsAlt + 4 * kMax);
constexpr size_t kOffStatus = align256(kOffHist + 4 * 256 * kMaxPasses);
constexpr size_t kOffTile = align256(kOffStatus + 4 * 256 * kMaxTiles * kMaxPasses);
constexpr size_t kOffErr = align256(kOffTile + 4 * kMaxPasses);
constexpr size_t kBytes = align256(kOffErr + 4);
static_assert(kBytes == JT_STATIC_SORT_BYTES, "JT_STATIC_SORT_BYTES must match the layout");

static __device__ __align__(256) unsigned char g_sort_scratch[kBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_addr[kMaxDevices] = {};

// The array's address on the current device (looked up once per device).
int scratch_address(void** out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return JT_ECUDA;
    if (dev >= kMaxDevices) return JT_EINVAL;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_sort_scratch) != cudaSuccess || !p) return JT_ECUDA;
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return JT_OK;
}

__device__ __forceinline__ uint32_t spread10_bits(uint32_t x)
{
    x &= 0x3FFu;
    x = (x | (x << 16)) & 0x030000FFu;
    x = (x | (x << 8)) & 0x0300F00Fu;
    x = (x | (x << 4)) & 0x030C30C3u;
    x = (x | (x << 2)) & 0x09249249u;
    return x;
}

// The reference's key of particle i from float3 positions:
// (morton30(x, y, z) << 32) | i with the quantisation of jt_debug_tree
// (scale 1024 / (2 box_half), no contraction, saturating float -> uint).
__global__ void k_morton_aos(const float* __restrict__ pos, int64_t n, float box_half,
                             uint64_t* __restrict__ key64, uint32_t* __restrict__ vals)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float scale = 1024.0f / (2.0f * box_half);
    float x = __fmul_rn(__fadd_rn(pos[3 * i], box_half), scale);
    float y = __fmul_rn(__fadd_rn(pos[3 * i + 1], box_half), scale);
    float z = __fmul_rn(__fadd_rn(pos[3 * i + 2], box_half), scale);
    uint32_t ix = min(__float2uint_rz(x), 0x3FFu);
    uint32_t iy = min(__float2uint_rz(y), 0x3FFu);
    uint32_t iz = min(__float2uint_rz(z), 0x3FFu);
    uint32_t m = spread10_bits(ix) | (spread10_bits(iy) << 1) | (spread10_bits(iz) << 2);
    key64[i] = ((uint64_t)m << 32) | (uint32_t)i;
    vals[i] = (uint32_t)i;
}

}  // namespace

extern "C" int jt_morton_sort_static(const float* pos, size_t n, double box_L, uint32_t* morton_out,
                                     int32_t* perm_out, void* stream)
{
    if (!pos || !morton_out || !perm_out || n == 0) return JT_EINVAL;
    if (n > (size_t)kMax) return JT_EINVAL;
    if (!(box_L > 0.0)) return JT_EINVAL;
    void* base = nullptr;
    int r = scratch_address(&base);
    if (r != JT_OK) return r;
    unsigned char* b = static_cast<unsigned char*>(base);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    uint64_t* key64 = reinterpret_cast<uint64_t*>(b + kOffKey);
    jt_sort_ws ws;
    ws.keys_alt = b + kOffKeyAlt;
    ws.vals = reinterpret_cast<uint32_t*>(b + kOffVals);
    ws.vals_alt = reinterpret_cast<uint32_t*>(b + kOffValsAlt);
    ws.hist = reinterpret_cast<uint32_t*>(b + kOffHist);
    ws.status = reinterpret_cast<uint32_t*>(b + kOffStatus);
    ws.tile_ctr = reinterpret_cast<uint32_t*>(b + kOffTile);
    ws.cap = kMax;
    ws.max_passes = kMaxPasses;
    unsigned* d_err = reinterpret_cast<unsigned*>(b + kOffErr);
    const int64_t nn = (int64_t)n;
    if (cudaMemsetAsync(d_err, 0, sizeof(unsigned), st) != cudaSuccess) return JT_ECUDA;
    k_morton_aos<<<(unsigned)((nn + 255) / 256), 256, 0, st>>>(pos, nn, (float)(box_L / 2.0), key64,
                                                                ws.vals);
    // the 30 Morton bits only: the keys start in index order and every LSD
    // pass is stable, so equal codes keep their index order (the low word)
    // without sorting its digits
    const int shifts[4] = {32, 40, 48, 56};
    r = jt_radix_sort_u64(key64, ws.vals, nn, shifts, 4, &ws, d_err, st);
    if (r != JT_OK) return r;
    jt_launch_split_keys(key64, nn, morton_out, reinterpret_cast<uint32_t*>(perm_out), st);
    if (cudaGetLastError() != cudaSuccess) return JT_ECUDA;
    unsigned e = 0;
    if (cudaMemcpyAsync(&e, d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, st) != cudaSuccess)
        return JT_ECUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return JT_ECUDA;
    return e ? JT_ETIMEDOUT : JT_OK;
}
