/*
 * Host-CPU emulation of the CUDA constructs used by the reference's kernel
 * source, so that the reference kernels themselves compile with g++ and run
 * on the CPU.  TEST INFRASTRUCTURE ONLY: this builds the checker that pins the
 * oracle restatements in oracle/*.c to the reference's own code.
 *
 * Execution model:
 *   - kernels without warp-level intrinsics run one thread after another
 *     (emu_launch_serial); atomics are then plain read-modify-writes;
 *   - warp-synchronous kernels run each warp as 32 fibers in lock-step
 *     (emu_launch_warps): every warp intrinsic is a rendezvous of the 32
 *     lanes, after which each lane gets the intrinsic's result.
 * Shared memory maps to thread_local storage (one OS thread runs a whole
 * block at a time, so it is shared by the block's lanes).
 */
#ifndef JANUS_CUDA_HOST_EMU_H
#define JANUS_CUDA_HOST_EMU_H

#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>

struct emu_uint3 { unsigned x, y, z; };
extern emu_uint3 threadIdx, blockIdx, blockDim, gridDim;

#define __global__
#define __device__ static inline
#define __host__
#define __restrict__ __restrict
#define __shared__ thread_local

/* ---- warp rendezvous (implemented in the harness) ---- */
enum { EMU_SHFL = 1, EMU_ALL = 2, EMU_BALLOT = 3, EMU_SYNCWARP = 4, EMU_BARRIER = 9 };
uint64_t emu_warp_sync(int kind, uint64_t value, int src_lane);
void emu_block_sync();

template <class T>
static inline T __shfl_sync(unsigned, T v, int src)
{
    uint64_t bits = 0;
    std::memcpy(&bits, &v, sizeof(T));
    uint64_t r = emu_warp_sync(EMU_SHFL, bits, src);
    T out;
    std::memcpy(&out, &r, sizeof(T));
    return out;
}
static inline int __all_sync(unsigned, int pred) { return (int)emu_warp_sync(EMU_ALL, pred != 0, 0); }
static inline unsigned __ballot_sync(unsigned, int pred) { return (unsigned)emu_warp_sync(EMU_BALLOT, pred != 0, 0); }
static inline void __syncwarp(unsigned = 0xFFFFFFFFu) { emu_warp_sync(EMU_SYNCWARP, 0, 0); }
/* block barrier: a rendezvous of all live threads of the block */
static inline void __syncthreads() { emu_block_sync(); }
static inline void __threadfence() {}

/* ---- atomics (serial or lock-step execution: plain RMW is exact) ---- */
static inline int atomicAdd(int* a, int v) { int o = *a; *a = o + v; return o; }
static inline unsigned atomicAdd(unsigned* a, unsigned v) { unsigned o = *a; *a = o + v; return o; }
static inline float atomicAdd(float* a, float v) { float o = *a; *a = o + v; return o; }
static inline unsigned long long atomicCAS(unsigned long long* a, unsigned long long cmp,
                                           unsigned long long v)
{
    unsigned long long o = *a;
    if (o == cmp) *a = v;
    return o;
}

/* ---- bit casts and integer intrinsics ---- */
static inline int __float_as_int(float f) { int i; std::memcpy(&i, &f, 4); return i; }
static inline float __int_as_float(int i) { float f; std::memcpy(&f, &i, 4); return f; }
static inline long long __double_as_longlong(double d) { long long i; std::memcpy(&i, &d, 8); return i; }
static inline double __longlong_as_double(long long i) { double d; std::memcpy(&d, &i, 8); return d; }
static inline int __popc(unsigned x) { return __builtin_popcount(x); }
static inline int __clzll(long long x) { return x ? __builtin_clzll((unsigned long long)x) : 64; }

/* CUDA's integer min/max overloads */
static inline unsigned min(unsigned a, unsigned b) { return a < b ? a : b; }
static inline unsigned max(unsigned a, unsigned b) { return a > b ? a : b; }
static inline int min(int a, int b) { return a < b ? a : b; }
static inline int max(int a, int b) { return a > b ? a : b; }

/* math: single-precision entry points the kernels call */
using std::sqrt;
static inline float rsqrtf(float x) { return 1.0f / std::sqrt(x); }

/* launches (implemented in the harness) */
void emu_launch_serial(unsigned grid, unsigned block, const std::function<void()>& body);
void emu_launch_warps(unsigned grid, unsigned block, const std::function<void()>& body);

#endif
