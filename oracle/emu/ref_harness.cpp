/*
 * Runs the reference's own CUDA kernels on the host CPU.  TEST INFRASTRUCTURE
 * ONLY: the result, oracle/_ref/libref_twopass.so, is the checker that pins the
 * C restatements in oracle/*.c; it is never linked into the product.
 *
 * The kernel text comes unmodified from the reference (see extract.py):
 *   twopass_kernels.cu  = CUDA_TWOPASS_KERNELS, src/nbody_gpu_twopass.rs:27-1813
 *   cufft_kernels.cu    = apply_green_kernel / normalize_kernel,
 *                         cuda/cufft_wrapper.cu:148-208, 290-295
 * The only host-side code restated here is the reference's 16-bit parameter
 * packing (src/nbody_gpu_twopass.rs:1932-1937, 4079-4082).
 */
#include "cuda_host_emu.h"
#include <cstdio>
#include <cstdlib>
#include <vector>

emu_uint3 threadIdx, blockIdx, blockDim, gridDim;

extern "C" {
/* dynamic shared memory named by the kernels (extern __shared__) */
thread_local int shared_stack[4096];
thread_local float sh_data[4096];
}

struct cufftDoubleComplex { double x, y; };

#include "twopass_kernels.cu"
#include "cufft_kernels.cu"

/* ------------------------------------------------------------------------ */
/* fibers: one per thread of the emulated block                              */
/* ------------------------------------------------------------------------ */
extern "C" void emu_ctx_switch(void** save_sp, void* new_sp);
__asm__(
    ".text\n"
    ".globl emu_ctx_switch\n"
    ".type emu_ctx_switch,@function\n"
    "emu_ctx_switch:\n"
    "  pushq %rbp\n  pushq %rbx\n  pushq %r12\n  pushq %r13\n  pushq %r14\n  pushq %r15\n"
    "  movq %rsp, (%rdi)\n"
    "  movq %rsi, %rsp\n"
    "  popq %r15\n  popq %r14\n  popq %r13\n  popq %r12\n  popq %rbx\n  popq %rbp\n"
    "  ret\n"
    ".size emu_ctx_switch, .-emu_ctx_switch\n");

namespace {
const size_t kStack = 256 * 1024;
struct Fib {
    void* sp;
    char* stack;
    int done;
    int kind;        /* 0 = runnable; EMU_* = waiting at a warp sync; 9 = block barrier */
    uint64_t val, res;
    int src;
};
std::vector<Fib> g_fib;
void* g_sched_sp;
int g_cur;
const std::function<void()>* g_body;
unsigned g_block;

void fiber_entry()
{
    (*g_body)();
    g_fib[g_cur].done = 1;
    emu_ctx_switch(&g_fib[g_cur].sp, g_sched_sp);
    std::abort();
}

void fiber_init(Fib& f)
{
    if (!f.stack) f.stack = (char*)std::malloc(kStack);
    uintptr_t top = ((uintptr_t)(f.stack + kStack)) & ~(uintptr_t)15;
    uint64_t* sp = (uint64_t*)top;
    *--sp = 0;                              /* fake return address slot (rsp = 8 mod 16 at entry) */
    *--sp = (uint64_t)(uintptr_t)&fiber_entry;
    for (int i = 0; i < 6; i++) *--sp = 0;  /* rbp rbx r12 r13 r14 r15 */
    f.sp = sp;
    f.done = 0; f.kind = 0;
}
}  // namespace

uint64_t emu_warp_sync(int kind, uint64_t value, int src_lane)
{
    Fib& f = g_fib[g_cur];
    f.kind = kind; f.val = value; f.src = src_lane;
    emu_ctx_switch(&f.sp, g_sched_sp);
    return f.res;
}

static int g_in_fibers = 0;

void emu_block_sync()
{
    if (!g_in_fibers) return;   /* serial launches run kernels without barriers */
    Fib& f = g_fib[g_cur];
    f.kind = EMU_BARRIER;
    emu_ctx_switch(&f.sp, g_sched_sp);
}

static void run_block(unsigned bx, unsigned block, const std::function<void()>& body)
{
    g_body = &body;
    g_block = block;
    if (g_fib.size() < block) g_fib.resize(block, Fib{nullptr, nullptr, 0, 0, 0, 0, 0});
    for (unsigned t = 0; t < block; t++) fiber_init(g_fib[t]);
    blockIdx = {bx, 0, 0};
    for (;;) {
        int progressed = 0, alive = 0;
        for (unsigned t = 0; t < block; t++) {
            Fib& f = g_fib[t];
            if (f.done || f.kind != 0) continue;
            g_cur = (int)t;
            threadIdx = {t, 0, 0};
            emu_ctx_switch(&g_sched_sp, f.sp);
            progressed = 1;
        }
        for (unsigned t = 0; t < block; t++) alive += !g_fib[t].done;
        if (!alive) break;
        /* resolve warp rendezvous: every live lane of the warp waits at one */
        for (unsigned w0 = 0; w0 < block; w0 += 32) {
            unsigned w1 = w0 + 32 < block ? w0 + 32 : block;
            int live = 0, waiting = 0, kind = -1, mixed = 0;
            for (unsigned t = w0; t < w1; t++) {
                Fib& f = g_fib[t];
                if (f.done) continue;
                live++;
                if (f.kind >= EMU_SHFL && f.kind <= EMU_SYNCWARP) {
                    waiting++;
                    if (kind < 0) kind = f.kind; else if (kind != f.kind) mixed = 1;
                }
            }
            if (!live || waiting != live) continue;
            if (mixed) { std::fprintf(stderr, "emu: divergent warp intrinsics\n"); std::abort(); }
            uint64_t all = 1, ballot = 0;
            for (unsigned t = w0; t < w1; t++) {
                Fib& f = g_fib[t];
                if (f.done) continue;
                all &= (f.val != 0);
                if (f.val) ballot |= 1ull << (t - w0);
            }
            for (unsigned t = w0; t < w1; t++) {
                Fib& f = g_fib[t];
                if (f.done) continue;
                if (kind == EMU_SHFL) {
                    unsigned s = w0 + (unsigned)(f.src & 31);
                    f.res = (s < w1) ? g_fib[s].val : 0;
                } else if (kind == EMU_ALL) f.res = all;
                else if (kind == EMU_BALLOT) f.res = ballot;
                else f.res = 0;
                f.kind = 0;
            }
            progressed = 1;
        }
        /* block barrier: every live thread waits at __syncthreads */
        {
            int live = 0, at_bar = 0;
            for (unsigned t = 0; t < block; t++) {
                if (g_fib[t].done) continue;
                live++;
                at_bar += g_fib[t].kind == EMU_BARRIER;
            }
            if (live && at_bar == live) {
                for (unsigned t = 0; t < block; t++)
                    if (!g_fib[t].done) g_fib[t].kind = 0;
                progressed = 1;
            }
        }
        if (!progressed) { std::fprintf(stderr, "emu: deadlock\n"); std::abort(); }
    }
}

void emu_launch_warps(unsigned grid, unsigned block, const std::function<void()>& body)
{
    gridDim = {grid, 1, 1};
    blockDim = {block, 1, 1};
    g_in_fibers = 1;
    for (unsigned b = 0; b < grid; b++) run_block(b, block, body);
    g_in_fibers = 0;
}

void emu_launch_serial(unsigned grid, unsigned block, const std::function<void()>& body)
{
    gridDim = {grid, 1, 1};
    blockDim = {block, 1, 1};
    for (unsigned b = 0; b < grid; b++) {
        blockIdx = {b, 0, 0};
        for (unsigned t = 0; t < block; t++) {
            threadIdx = {t, 0, 0};
            body();
        }
    }
}

static unsigned blocks_for(long long n, unsigned bs) { return (unsigned)((n + bs - 1) / bs); }

/* ------------------------------------------------------------------------ */
/* C API over the reference kernels                                          */
/* ------------------------------------------------------------------------ */
extern "C" {

/* compute_morton_f32: keys (m30 << 32) | idx */
void ref_morton(const float* pos, int n, float box_half, unsigned long long* keys, int* idx)
{
    float inv_cell = 0.0f; /* unused by the kernel */
    emu_launch_serial(blocks_for(n, 256), 256, [&] {
        compute_morton_f32(pos, keys, idx, n, box_half, inv_cell);
    });
}

/* the reference's radix sort: 8 passes x (histogram, prefix, scatter) */
void ref_radix_sort(unsigned long long* keys, int* vals, int n)
{
    unsigned nb = blocks_for(n, 256);
    std::vector<unsigned long long> k2(n);
    std::vector<int> v2(n);
    std::vector<unsigned> hist((size_t)nb * 256), glob(256);
    for (int pass = 0; pass < 8; pass++) {
        int shift = pass * 8;
        unsigned long long* kin = (pass % 2 == 0) ? keys : k2.data();
        unsigned long long* kout = (pass % 2 == 0) ? k2.data() : keys;
        int* vin = (pass % 2 == 0) ? vals : v2.data();
        int* vout = (pass % 2 == 0) ? v2.data() : vals;
        emu_launch_warps(nb, 256, [&] { radix_histogram(kin, hist.data(), n, shift); });
        emu_launch_warps(1, 256, [&] { radix_prefix_sum(hist.data(), glob.data(), (int)nb); });
        emu_launch_warps(nb, 256, [&] {
            radix_scatter(kin, kout, vin, vout, hist.data(), glob.data(), n, shift);
        });
    }
}

/* build_bvh_tp over sorted keys; parent must be preset to -1 by the caller
 * (set_i32 in build_single_sign_tree) */
void ref_karras(const unsigned long long* keys, int n, int* left, int* right,
                int* parent, int* rl, int* rr)
{
    if (n < 2) return;
    emu_launch_serial(blocks_for(n - 1, 256), 256, [&] {
        build_bvh_tp(keys, left, right, parent, rl, rr, n);
    });
}

/* init_leaves_tp + reduce_tp; node_mass/types/atomic zeroed as the host does */
void ref_leaves_reduce(const float* pos_sorted, int n, float box_half, float mass_factor,
                       const int* left, const int* right, const int* parent,
                       const int* rl, const int* rr, float* node_pos,
                       float* node_mass, int* types)
{
    int nn = 2 * n - 1;
    std::vector<int> atom(nn, 0);
    for (int i = 0; i < nn; i++) { node_mass[i] = 0.0f; types[i] = 0; }
    emu_launch_serial(blocks_for(n, 256), 256, [&] {
        init_leaves_tp(pos_sorted, node_pos, node_mass, types, atom.data(), n, box_half, mass_factor);
    });
    emu_launch_serial(blocks_for(n, 256), 256, [&] {
        reduce_tp(left, right, parent, rl, rr, node_pos, node_mass, types, atom.data(), n, box_half);
    });
}

void ref_cic_scatter(const float* pos, const signed char* signs, double* rho_plus,
                     double* rho_minus, int n, int grid, float box_half, float inv_cell)
{
    emu_launch_serial(blocks_for(n, 256), 256, [&] {
        cic_scatter(pos, signs, rho_plus, rho_minus, n, grid, box_half, inv_cell);
    });
}

void ref_cic_gather(const float* pos, const signed char* signs, const double* phi_plus,
                    const double* phi_minus, float* pm_forces, int n, int grid,
                    float box_half, float inv_cell, float cell)
{
    emu_launch_serial(blocks_for(n, 256), 256, [&] {
        cic_gather(pos, signs, phi_plus, phi_minus, pm_forces, n, grid, box_half, inv_cell, cell);
    });
}

/* apply_green_kernel on a D2Z half spectrum nx*ny*(nz/2+1) (interleaved re,im) */
void ref_apply_green(double* data, int nx, int ny, int nz, double dk, double g_constant,
                     double r_s, int k_min)
{
    long long total = (long long)nx * ny * (nz / 2 + 1);
    cufftDoubleComplex* d = (cufftDoubleComplex*)data;
    emu_launch_serial(blocks_for(total, 256), 256, [&] {
        apply_green_kernel(d, nx, ny, nz, dk, g_constant, r_s, k_min);
    });
}

void ref_normalize(double* data, int n, double factor)
{
    emu_launch_serial(blocks_for(n, 256), 256, [&] { normalize_kernel(data, n, factor); });
}

/* host packing of compute_short_range_forces (:4079-4082) and pack_rcut_boxhalf
 * (:1932-1937); Rust `as u32` saturates */
static unsigned sat_u32(double v) { return v <= 0.0 ? 0u : (v >= 4294967295.0 ? 0xFFFFFFFFu : (unsigned)v); }

void ref_pack_params(double theta, double softening, double r_cut, double box_size,
                     float* theta_soft_packed, float* rcut_boxhalf_packed)
{
    unsigned ti = sat_u32(theta * 1000.0), si = sat_u32(softening * 1000.0);
    if (ti > 0xFFFF) ti = 0xFFFF;
    if (si > 0xFFFF) si = 0xFFFF;
    unsigned a = (ti << 16) | si;
    unsigned ri = sat_u32(r_cut), bi = sat_u32(box_size / 2.0);
    if (ri > 0xFFFF) ri = 0xFFFF;
    if (bi > 0xFFFF) bi = 0xFFFF;
    unsigned b = (ri << 16) | bi;
    std::memcpy(theta_soft_packed, &a, 4);
    std::memcpy(rcut_boxhalf_packed, &b, 4);
}

/* forces_treepm_short_range: 256 threads/block, 4096 B dynamic shared memory */
void ref_short_range(const float* pos_all, const signed char* signs_all,
                     const float* node_pos, const float* node_mass, const int* left,
                     const int* right, const int* types, float* acc, int n_all_signed,
                     float theta_soft_packed, float rcut_boxhalf_packed)
{
    int n = n_all_signed > 0 ? n_all_signed : -n_all_signed;
    emu_launch_warps(blocks_for(n, 256), 256, [&] {
        forces_treepm_short_range(pos_all, signs_all, node_pos, node_mass, left, right,
                                  types, acc, n_all_signed, theta_soft_packed,
                                  rcut_boxhalf_packed);
    });
}

/* host packing of the screened branch of compute_short_range_forces
 * (:4008-4016): theta and softening ROUNDED to 1e-3 (f64::round, half away
 * from zero) before the saturating cast; lambda(z) = lambda_0 sqrt(1 + z)
 * and box_half by pack_lambda_boxhalf (:1921-1927), truncated. */
void ref_pack_screening(double theta, double softening, double lambda_0, double z, double box_size,
                        float* theta_soft_packed, float* lambda_boxhalf_packed)
{
    unsigned ti = sat_u32(std::round(theta * 1000.0)), si = sat_u32(std::round(softening * 1000.0));
    if (ti > 0xFFFF) ti = 0xFFFF;
    if (si > 0xFFFF) si = 0xFFFF;
    unsigned a = (ti << 16) | si;
    double lz = lambda_0 * std::sqrt(1.0 + z);
    unsigned li = sat_u32(lz * 10.0), bi = sat_u32(box_size / 2.0);
    if (li > 0xFFFF) li = 0xFFFF;
    if (bi > 0xFFFF) bi = 0xFFFF;
    unsigned b = (li << 16) | bi;
    std::memcpy(theta_soft_packed, &a, 4);
    std::memcpy(lambda_boxhalf_packed, &b, 4);
}

/* forces_twopass_warpcoherent_screening: 256 threads/block, 4096 B dynamic
 * shared memory, as compute_short_range_forces launches it (:4036-4073) */
void ref_screening(const float* pos_all, const signed char* signs_all, const float* node_pos,
                   const float* node_mass, const int* left, const int* right, const int* types,
                   float* acc, int n_all, int tree_sign, float theta_soft_packed,
                   float lambda_boxhalf_packed)
{
    emu_launch_warps(blocks_for(n_all, 256), 256, [&] {
        forces_twopass_warpcoherent_screening(pos_all, signs_all, node_pos, node_mass, left, right,
                                              types, acc, n_all, tree_sign, theta_soft_packed,
                                              lambda_boxhalf_packed);
    });
}

void ref_drift(float* pos, const float* vel, float dt, float box_half, int n)
{
    emu_launch_serial(blocks_for(n, 256), 256, [&] { drift_f32(pos, vel, dt, box_half, n); });
}

void ref_kick(float* vel, const float* acc, float dt, int n, float hubble, float dtau)
{
    emu_launch_serial(blocks_for(n, 256), 256, [&] { kick_f32(vel, acc, dt, n, hubble, dtau); });
}

}  // extern "C"
