/*
 * Replays the reference's GPU TreePM step on the device, with the
 * reference's own kernels.  TEST INFRASTRUCTURE ONLY: a timing yardstick (the
 * reference GPU path recompiled for sm_100a), never linked into the product.
 *
 * The kernel text comes unmodified from the reference (oracle/emu/extract.py):
 *   twopass_kernels.cu = CUDA_TWOPASS_KERNELS, src/nbody_gpu_twopass.rs:27-1813
 *   cufft_kernels.cu   = apply_green_kernel / normalize_kernel,
 *                        cuda/cufft_wrapper.cu:148-208, 290-295
 * This file restates only the host side: the launch sequence, launch shapes,
 * parameter packing and device synchronisations of
 *   step_treepm_gpu            (src/nbody_gpu_twopass.rs:4486-4649)
 *   compute_short_range_forces (:3961-4138, the unscreened branch)
 *   build_single_sign_tree     (:2338-2545)
 *   cufft_solve_device         (cuda/cufft_wrapper.cu:336-398: D2D copy, D2Z,
 *                               Green's function, Z2D, normalisation)
 * with double-precision PM grids of any power-of-two size (the reference
 * hard-wires 256^3, :2098, :2257).
 */
#include <cuda_runtime.h>
#include <cufft.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "twopass_kernels.cu"
#include "cufft_kernels.cu"

namespace {

struct State {
    int n = 0, n_pos = 0, n_neg = 0, grid = 0;
    double box = 0, theta = 0, soft = 0, mass_factor = 0;
    float *pos = nullptr, *vel = nullptr, *acc = nullptr, *pm = nullptr;
    signed char* signs = nullptr;
    double *rho_p = nullptr, *rho_m = nullptr, *phi_p = nullptr, *phi_m = nullptr;
    cufftDoubleComplex* kspace = nullptr;
    cufftHandle r2c = 0, c2r = 0;
    float *pos_sign = nullptr, *pos_sign_tmp = nullptr;
    int *idx_map = nullptr, *idx_map_tmp = nullptr;
    unsigned long long *morton = nullptr, *morton_tmp = nullptr;
    int *sorted = nullptr, *sorted_tmp = nullptr;
    unsigned *hist = nullptr, *glob = nullptr;
    int *left = nullptr, *right = nullptr, *parent = nullptr, *rl = nullptr, *rr = nullptr;
    float *node_pos = nullptr, *node_mass = nullptr;
    int *types = nullptr, *atom = nullptr, *count = nullptr;
    double t_pm_ms = 0, t_bh_ms = 0, t_other_ms = 0;
};
State g;

unsigned blocks(long long n) { return (unsigned)((n + 255) / 256); }

// Rust `as u32` saturates; the packing of :4079-4082 and :1932-1937
unsigned sat_u32(double v) { return v <= 0.0 ? 0u : (v >= 4294967295.0 ? 0xFFFFFFFFu : (unsigned)v); }

float bits_to_float(unsigned b)
{
    float f;
    std::memcpy(&f, &b, 4);
    return f;
}

#define CK(x)                                  \
    do {                                       \
        if ((x) != cudaSuccess) return -3;     \
    } while (0)

int solve_device(double* rho, double* phi, double g_constant, double r_s)
{
    const int M = g.grid;
    const long long n_real = (long long)M * M * M, n_complex = (long long)M * M * (M / 2 + 1);
    CK(cudaMemcpy(phi, rho, n_real * sizeof(double), cudaMemcpyDeviceToDevice));
    if (cufftExecD2Z(g.r2c, phi, g.kspace) != CUFFT_SUCCESS) return -3;
    CK(cudaDeviceSynchronize());
    const double dk = 2.0 * 3.14159265358979323846 / g.box;
    apply_green_kernel<<<blocks(n_complex), 256>>>(g.kspace, M, M, M, dk, g_constant, r_s, 0);
    CK(cudaDeviceSynchronize());
    if (cufftExecZ2D(g.c2r, g.kspace, phi) != CUFFT_SUCCESS) return -3;
    CK(cudaDeviceSynchronize());
    normalize_kernel<<<blocks(n_real), 256>>>(phi, (int)n_real, 1.0 / (double)n_real);
    CK(cudaDeviceSynchronize());
    return 0;
}

int build_single_sign_tree(int n)
{
    const float box_half = (float)(g.box / 2.0);
    const float inv_cell = (float)(2097152.0 / g.box);
    const int n_nodes = 2 * n - 1;
    compute_morton_f32<<<blocks(n), 256>>>(g.pos_sign, g.morton, g.sorted, n, box_half, inv_cell);
    CK(cudaDeviceSynchronize());
    const int nb = (int)blocks(n);
    for (int pass = 0; pass < 8; pass++) {
        const int shift = pass * 8;
        unsigned long long* kin = pass % 2 == 0 ? g.morton : g.morton_tmp;
        unsigned long long* kout = pass % 2 == 0 ? g.morton_tmp : g.morton;
        int* vin = pass % 2 == 0 ? g.sorted : g.sorted_tmp;
        int* vout = pass % 2 == 0 ? g.sorted_tmp : g.sorted;
        radix_histogram<<<nb, 256>>>(kin, g.hist, n, shift);
        radix_prefix_sum<<<1, 256>>>(g.hist, g.glob, nb);
        radix_scatter<<<nb, 256>>>(kin, kout, vin, vout, g.hist, g.glob, n, shift);
    }
    CK(cudaDeviceSynchronize());
    reorder_f32x3<<<blocks(n), 256>>>(g.pos_sign, g.pos_sign_tmp, g.sorted, n);
    std::swap(g.pos_sign, g.pos_sign_tmp);
    reorder_i32<<<blocks(n), 256>>>(g.idx_map, g.idx_map_tmp, g.sorted, n);
    std::swap(g.idx_map, g.idx_map_tmp);
    CK(cudaDeviceSynchronize());
    reset_i32<<<blocks(n_nodes), 256>>>(g.atom, n_nodes);
    reset_i32<<<blocks(n_nodes), 256>>>(g.types, n_nodes);
    reset_f32<<<blocks(n_nodes), 256>>>(g.node_mass, n_nodes);
    set_i32<<<blocks(n_nodes), 256>>>(g.parent, n_nodes, -1);
    CK(cudaDeviceSynchronize());
    if (n > 1) build_bvh_tp<<<blocks(n - 1), 256>>>(g.morton, g.left, g.right, g.parent, g.rl, g.rr, n);
    CK(cudaDeviceSynchronize());
    init_leaves_tp<<<blocks(n), 256>>>(g.pos_sign, g.node_pos, g.node_mass, g.types, g.atom, n, box_half,
                                       (float)g.mass_factor);
    CK(cudaDeviceSynchronize());
    reduce_tp<<<blocks(n), 256>>>(g.left, g.right, g.parent, g.rl, g.rr, g.node_pos, g.node_mass, g.types,
                                  g.atom, n, box_half);
    CK(cudaDeviceSynchronize());
    return 0;
}

int short_range(double r_cut)
{
    const int n = g.n;
    reset_f32<<<blocks(3LL * n), 256>>>(g.acc, n * 3);
    CK(cudaDeviceSynchronize());
    unsigned ti = sat_u32(g.theta * 1000.0), si = sat_u32(g.soft * 1000.0);
    ti = ti > 0xFFFF ? 0xFFFF : ti;
    si = si > 0xFFFF ? 0xFFFF : si;
    const float ts_packed = bits_to_float((ti << 16) | si);
    unsigned ri = sat_u32(r_cut), bi = sat_u32(g.box / 2.0);
    ri = ri > 0xFFFF ? 0xFFFF : ri;
    bi = bi > 0xFFFF ? 0xFFFF : bi;
    const float rb_packed = bits_to_float((ri << 16) | bi);
    for (int sign : {1, -1}) {
        reset_i32<<<1, 1>>>(g.count, 1);
        extract_by_sign<<<blocks(n), 256>>>(g.pos, g.signs, g.pos_sign, g.idx_map, n, sign, g.count);
        CK(cudaDeviceSynchronize());
        const int ns = sign > 0 ? g.n_pos : g.n_neg;
        if (ns > 0) {
            int r = build_single_sign_tree(ns);
            if (r) return r;
            forces_treepm_short_range<<<blocks(n), 256, 4096>>>(
                g.pos, g.signs, g.node_pos, g.node_mass, g.left, g.right, g.types, g.acc,
                sign > 0 ? n : -n, ts_packed, rb_packed);
            CK(cudaDeviceSynchronize());
        }
    }
    return 0;
}

template <class T>
int dal(T** p, size_t count)
{
    return cudaMalloc((void**)p, sizeof(T) * (count ? count : 1)) == cudaSuccess ? 0 : -2;
}

}  // namespace

extern "C" {

void rg_free()
{
    void* ptrs[] = {g.pos, g.vel, g.acc, g.pm, g.signs, g.rho_p, g.rho_m, g.phi_p, g.phi_m, g.kspace,
                    g.pos_sign, g.pos_sign_tmp, g.idx_map, g.idx_map_tmp, g.morton, g.morton_tmp,
                    g.sorted, g.sorted_tmp, g.hist, g.glob, g.left, g.right, g.parent, g.rl, g.rr,
                    g.node_pos, g.node_mass, g.types, g.atom, g.count};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (g.r2c) cufftDestroy(g.r2c);
    if (g.c2r) cufftDestroy(g.c2r);
    g = State();
}

/* Load n particles (host AoS float3 positions and velocities, i8 signs) into
 * a box of side `box` with a grid^3 PM mesh; every particle carries
 * mass_factor (the reference's convention). */
int rg_init(int n, const float* pos, const float* vel, const signed char* signs, int grid, double box,
            double theta, double softening, double mass_factor)
{
    rg_free();
    if (n <= 0 || grid < 8 || (grid & (grid - 1))) return -1;
    g.n = n;
    g.grid = grid;
    g.box = box;
    g.theta = theta;
    g.soft = softening;
    g.mass_factor = mass_factor;
    for (int i = 0; i < n; i++) (signs[i] > 0 ? g.n_pos : g.n_neg)++;
    // radix_scatter (:1549-1636) calls full-warp __ballot_sync/__shfl_sync
    // inside `if (tid < n)`: a partial last warp would leave named lanes out
    // of the sync, so only species counts that fill whole blocks are replayed
    if (g.n_pos % 256 || g.n_neg % 256) {
        g = State();
        return -1;
    }
    const long long G = (long long)grid * grid * grid, Gc = (long long)grid * grid * (grid / 2 + 1);
    const int nodes = 2 * n;
    int r = 0;
    r |= dal(&g.pos, 3LL * n); r |= dal(&g.vel, 3LL * n); r |= dal(&g.acc, 3LL * n); r |= dal(&g.pm, 3LL * n);
    r |= dal(&g.signs, n);
    r |= dal(&g.rho_p, G); r |= dal(&g.rho_m, G); r |= dal(&g.phi_p, G); r |= dal(&g.phi_m, G);
    r |= dal(&g.kspace, Gc);
    r |= dal(&g.pos_sign, 3LL * n); r |= dal(&g.pos_sign_tmp, 3LL * n);
    r |= dal(&g.idx_map, n); r |= dal(&g.idx_map_tmp, n);
    r |= dal(&g.morton, n); r |= dal(&g.morton_tmp, n); r |= dal(&g.sorted, n); r |= dal(&g.sorted_tmp, n);
    r |= dal(&g.hist, (size_t)blocks(n) * 256); r |= dal(&g.glob, 256);
    r |= dal(&g.left, nodes); r |= dal(&g.right, nodes); r |= dal(&g.parent, nodes);
    r |= dal(&g.rl, nodes); r |= dal(&g.rr, nodes);
    r |= dal(&g.node_pos, 7LL * nodes); r |= dal(&g.node_mass, nodes);
    r |= dal(&g.types, nodes); r |= dal(&g.atom, nodes); r |= dal(&g.count, 1);
    if (r) {
        rg_free();
        return -2;
    }
    if (cudaMemcpy(g.pos, pos, sizeof(float) * 3 * n, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(g.vel, vel, sizeof(float) * 3 * n, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(g.signs, signs, n, cudaMemcpyHostToDevice) != cudaSuccess)
        return -3;
    if (cufftPlan3d(&g.r2c, grid, grid, grid, CUFFT_D2Z) != CUFFT_SUCCESS ||
        cufftPlan3d(&g.c2r, grid, grid, grid, CUFFT_Z2D) != CUFFT_SUCCESS)
        return -3;
    return 0;
}

/* One step_treepm_gpu(dt, r_cut, hubble, dtau_per_dt); *ms = device time of
 * the whole step (CUDA events), pm_ms / bh_ms its PM and short-range parts. */
int rg_step(double dt, double r_cut, double hubble, double dtau_per_dt, double* ms, double* pm_ms,
            double* bh_ms)
{
    const int n = g.n, grid = g.grid;
    const long long G = (long long)grid * grid * grid;
    const float box_half = (float)(g.box / 2.0);
    const float half_dt = (float)(dt / 2.0);
    const float cell = (float)(g.box / grid), inv_cell = (float)(grid / g.box);
    const double cell_vol = (g.box / grid) * (g.box / grid) * (g.box / grid);
    const double g_constant = g.mass_factor / cell_vol;
    cudaEvent_t e0, e1, e2, e3;
    cudaEventCreate(&e0); cudaEventCreate(&e1); cudaEventCreate(&e2); cudaEventCreate(&e3);
    cudaEventRecord(e0);
    drift_f32<<<blocks(n), 256>>>(g.pos, g.vel, half_dt, box_half, n);
    CK(cudaDeviceSynchronize());
    cudaEventRecord(e1);
    reset_f64_grid<<<blocks(G), 256>>>(g.rho_p, (int)G);
    reset_f64_grid<<<blocks(G), 256>>>(g.rho_m, (int)G);
    CK(cudaDeviceSynchronize());
    cic_scatter<<<blocks(n), 256>>>(g.pos, g.signs, g.rho_p, g.rho_m, n, grid, box_half, inv_cell);
    CK(cudaDeviceSynchronize());
    const double r_s = r_cut / 3.0;
    int r = solve_device(g.rho_p, g.phi_p, g_constant, r_s);
    if (!r) r = solve_device(g.rho_m, g.phi_m, g_constant, r_s);
    if (r) return r;
    cic_gather<<<blocks(n), 256>>>(g.pos, g.signs, g.phi_p, g.phi_m, g.pm, n, grid, box_half, inv_cell, cell);
    CK(cudaDeviceSynchronize());
    cudaEventRecord(e2);
    r = short_range(r_cut);
    if (r) return r;
    cudaEventRecord(e3);
    add_pm_forces<<<blocks(n), 256>>>(g.acc, g.pm, n);
    CK(cudaDeviceSynchronize());
    kick_f32<<<blocks(n), 256>>>(g.vel, g.acc, (float)dt, n, (float)hubble, (float)dtau_per_dt);
    CK(cudaDeviceSynchronize());
    drift_f32<<<blocks(n), 256>>>(g.pos, g.vel, half_dt, box_half, n);
    CK(cudaDeviceSynchronize());
    cudaEvent_t e4;
    cudaEventCreate(&e4);
    cudaEventRecord(e4);
    CK(cudaEventSynchronize(e4));
    float a = 0, b = 0, c = 0;
    cudaEventElapsedTime(&a, e0, e4);
    cudaEventElapsedTime(&b, e1, e2);
    cudaEventElapsedTime(&c, e2, e3);
    if (ms) *ms = a;
    if (pm_ms) *pm_ms = b;
    if (bh_ms) *bh_ms = c;
    cudaEventDestroy(e0); cudaEventDestroy(e1); cudaEventDestroy(e2); cudaEventDestroy(e3);
    cudaEventDestroy(e4);
    return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

/* positions and velocities back (host AoS float3) */
int rg_get(float* pos, float* vel)
{
    if (pos && cudaMemcpy(pos, g.pos, sizeof(float) * 3 * g.n, cudaMemcpyDeviceToHost) != cudaSuccess) return -3;
    if (vel && cudaMemcpy(vel, g.vel, sizeof(float) * 3 * g.n, cudaMemcpyDeviceToHost) != cudaSuccess) return -3;
    return 0;
}

}  // extern "C"
