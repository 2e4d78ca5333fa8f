// Internal declarations of the B200 TreePM engine (sm_100a).
//
// Device layout (per species s = 0 for m+, 1 for m-; n_s particles):
//   particles, kept in Morton order of the last tree build:
//     pos[s]  float4 (x, y, z, 0)        vel[s] float4 (vx, vy, vz, 0)
//     acc[s]  float4 (ax, ay, az, 0)     id[s]  int (index in the caller's
//                                               species array)
//   tree of species s, 2 n_s - 1 nodes in the Karras numbering (internal
//   0..n_s-2, leaf j at n_s-1+j, leaf j = sorted particle j):
//     child  int2   (left, right)        parent int
//     com    float4 (com x, y, z, mass)
//     bmin, bmax float4 tight AABB (ACCURATE) or (cx,cy,cz,hs) cube in bmin
//                   (RCOMPAT, the reference's node geometry)
//     quad0  float4 (Qxx, Qyy, Qzz, Qxy), quad1 float2 (Qxz, Qyz): second
//                   central moments sum m d d^T (ACCURATE)
//   PM grid (M^3 cells, index x + M (y + M z), nodes at -L/2 + i h):
//     rho float (signed source s m / h^3), rho_k complex M^2 (M/2+1),
//     force_k 3 x complex, force 3 x float M^3 (acceleration of an m+
//     particle; an m- particle gets the negative).
#pragma once
#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>

#include <string>

#include "../../include/janus_treepm.h"

#define JT_WARPS_PER_BLOCK 4

// device-side error bits (jt_handle::d_err)
#define JT_ERRBIT_STACK     1u   // walk stack overflow
#define JT_ERRBIT_LOOKBACK  2u   // radix look-back wait gave up
#define JT_ERRBIT_LIST      4u   // interaction list overflow

struct jt_tree_dev {
    int64_t n;         // particles (leaves)
    int2* child;
    int2* range;       // internal node i: sorted particle range [first, last]
    int* parent;
    int* flag;         // arrival counters for the bottom-up pass
    float4* com;
    float4* bmin;
    float4* bmax;
    float4* quad0;
    float2* quad1;
    uint32_t* m30;     // sorted Morton codes (Karras keys, high word)
    uint32_t* tie;     // low word of the Karras key (caller index or position)
};

struct jt_sort_ws {
    // onesweep workspace, sized for the largest species
    void* keys_alt;       // key ping-pong (u32 or u64)
    uint32_t* vals;       // permutation (values)
    uint32_t* vals_alt;
    uint32_t* hist;       // [max_passes][256] global digit counts -> bases
    uint32_t* status;     // [max_passes][num_tiles][256] look-back words
    uint32_t* tile_ctr;   // [max_passes]
    int64_t cap;          // elements
    int max_passes;
};

// ---------------------------------------------------------------- batches
// A batch advances several independent boxes with ONE launch per stage.
// Work is described by segments (one per box and species) and boxes; every
// batched kernel maps its flattened work items (particles, tiles, nodes,
// 32-particle groups) to a segment or box through an exclusive prefix table
// (jt_find: binary search, log2(#segments) steps).  A single box is the batch
// of one (two segments).
struct jt_seg_dev {
    float4* pos;          // state, Morton order of the last build
    float4* vel;
    float4* acc;
    float4* pos_b;        // reorder targets (swapped after each build)
    float4* vel_b;
    int* id;
    int* id_b;
    int64_t n;
    jt_tree_dev tree;     // tree.m30 doubles as the sort key array
    uint32_t* vals;       // sort values (permutation) and its ping-pong
    uint32_t* vals_alt;
    uint32_t* keys_alt;
    uint32_t* hist;       // [4][256] digit counts -> bases
    uint32_t* status;     // [4][tiles][256] look-back words
    int box;              // owning box
    int species;          // 0 = m+, 1 = m-
};

struct jt_box_dev {
    float L, halfL, h_inv;
    float rc2, eps2, c, theta2;
    float mass[2];
    float box_half;       // float(L/2), the reference's Morton box_half
    float kick_drag;      // H * dtau of the current step
    float dt;             // step of this box (kicks and drifts take a fraction of it)
    int M, order, ngrid;
    int T, tile_shift, ntiles;
    float* rho;           // ngrid grids
    float2* rho_k;        // ngrid spectra
    float2* force_k;      // 3*ngrid spectra
    const float4* tabs;   // 2*M per-axis k tables
    float* force;         // 3*ngrid force grids
    int4* ranges;         // per-tile particle ranges of both species
    int seg[2];           // segment index of each species (-1: none)
    // Yukawa screening of opposite-species pairs (kappa > 0): the unsigned
    // source S = rho+ + rho- on its own grids (rho_s ...), the signed source D
    // takes the Green's function (G_N + G_Y) / 2 and S (G_N - G_Y) / 2, and
    // an m+/m- particle takes s A_D + A_S; cross pairs of the short range
    // read ytab (the Yukawa split factor) instead of the Newtonian table
    float ky2;            // kappa^2 (0: no screening)
    float yfac;           // exp(-kappa^2 r_s^2)
    float* rho_s;
    float2* rho_s_k;
    float2* force_s_k;
    float* force_s;
    const float2* ytab;   // the Yukawa kernel's log table (JT_LTAB_N entries)
    int nb;               // cells per axis of the near-field cell list (0: tree walk only)
    int cell_kmax;        // a cell whose 27-cell neighbourhood holds more goes to the tree walk
    float cell_inv;       // nb / L
    int64_t cbase;        // this box's first cell in the pass's cell tables
};

__device__ __forceinline__ int jt_find(const int64_t* __restrict__ prefix, int count, int64_t i)
{
    // largest b with prefix[b] <= i (prefix[0] = 0, prefix[count] = total)
    int lo = 0, hi = count - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= i) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// ---------------------------------------------------------------- math
// Short-range factor of the Gaussian split (potential erfc(r/2r_s)/r):
//   S(x) = erfc(x) + (2/sqrt(pi)) x exp(-x^2),  x = r / (2 r_s).
// erfc(x) from Abramowitz & Stegun 7.1.26 (absolute error <= 1.5e-7):
//   erfc(x) = t (a1 + t (a2 + t (a3 + t (a4 + t a5)))) exp(-x^2), t = 1/(1 + p x).
struct jt_sfac { float S, dS, d2S; };

__device__ __forceinline__ float jt_erfc_as(float x, float e)
{
    const float p = 0.3275911f;
    const float a1 = 0.254829592f, a2 = -0.284496736f, a3 = 1.421413741f,
                a4 = -1.453152027f, a5 = 1.061405429f;
    float t = __fdividef(1.0f, fmaf(p, x, 1.0f));   // fast reciprocal; t in (0, 1]
    float poly = fmaf(t, fmaf(t, fmaf(t, fmaf(t, a5, a4), a3), a2), a1);
    return t * poly * e;
}

// S(x) only (pair interactions); e = exp(-x^2)
__device__ __forceinline__ float jt_split_S(float x)
{
    float e = __expf(-x * x);
    return jt_erfc_as(x, e) + 1.1283791671f * x * e;
}

// S and its first two derivatives with respect to r (c = 1/(2 r_s)):
//   S'  = -(4/sqrt(pi)) c x^2 e,  S'' = -(8/sqrt(pi)) c^2 x e (1 - x^2)
__device__ __forceinline__ jt_sfac jt_split_S2(float x, float c)
{
    float e = __expf(-x * x);
    jt_sfac s;
    s.S = jt_erfc_as(x, e) + 1.1283791671f * x * e;
    s.dS = -2.2567583342f * c * x * x * e;
    s.d2S = -4.5135166684f * c * c * x * e * (1.0f - x * x);
    return s;
}

// Mass-assignment stencil along one axis at grid coordinate g (nodes at
// integers): returns the first node index and fills ORDER weights.
//   ORDER 2 (CIC): nodes floor(g), +1; weights 1-f, f
//   ORDER 3 (TSC): nodes c-1, c, c+1 with c = nearest node, d = g - c;
//                  weights (1/2)(1/2-d)^2, 3/4-d^2, (1/2)(1/2+d)^2
//   ORDER 4 (PCS, the cubic B-spline): nodes f-1 .. f+2 with f = floor(g),
//                  t = g - f, s = 1 - t; weights s^3/6, 2/3 - t^2 + t^3/2,
//                  2/3 - s^2 + s^3/2, t^3/6
// Deposit and interpolation use the same stencil, so the scheme exerts no
// self-force and conserves momentum.
template <int ORDER>
__device__ __forceinline__ int jt_stencil(float g, float* w)
{
    if (ORDER == 2) {
        float f0 = floorf(g);
        float f = g - f0;
        w[0] = 1.0f - f;
        w[1] = f;
        return (int)f0;
    } else if (ORDER == 4) {
        const float f0 = floorf(g);
        const float t = g - f0, s = 1.0f - t;
        const float t2 = t * t, s2 = s * s;
        w[0] = (1.0f / 6.0f) * s2 * s;
        w[1] = fmaf(0.5f * t2, t, 2.0f / 3.0f - t2);
        w[2] = fmaf(0.5f * s2, s, 2.0f / 3.0f - s2);
        w[3] = (1.0f / 6.0f) * t2 * t;
        return (int)f0 - 1;
    } else {
        float c = floorf(g + 0.5f);
        float d = g - c;
        w[0] = 0.5f * (0.5f - d) * (0.5f - d);
        w[1] = 0.75f - d * d;
        w[2] = 0.5f * (0.5f + d) * (0.5f + d);
        return (int)c - 1;
    }
}

__device__ __forceinline__ float jt_wrap(float d, float L, float halfL)
{
    // minimum image for |d| < 1.5 L
    d = (d > halfL) ? d - L : d;
    d = (d < -halfL) ? d + L : d;
    return d;
}

// Near-field cells whose 27-cell neighbourhood holds more candidates than
// this (at the config's r_cut; scaled by (cut / r_cut)^3 for a widened cut)
// send their targets to the tree walk: clustered data, where the dense
// evaluation's cost grows with the square of the local count.
#ifndef JT_CELL_KMAX
#define JT_CELL_KMAX 2048
#endif

// The short-range cut of an accurate-mode box: r_cut, or with cut_tail_ppm
// = k > 0 the radius where S(r / 2 r_s) = k * 1e-6 when that is larger.
double jt_short_cut(const jt_config& c);

// ---------------------------------------------------------------- launchers
// Raise a kernel's dynamic shared-memory limit to `bytes` on the current
// device.  cudaFuncSetAttribute applies to the device current when it runs,
// so the setting is kept per (device, kernel) under a lock (threads driving
// different devices, or the same one, may launch concurrently).
int jt_smem_attr(const void* kernel, int bytes);

// sort (jt_sort.cu)
int jt_sort_ws_alloc(jt_sort_ws* ws, int64_t cap, int max_passes);
void jt_sort_ws_free(jt_sort_ws* ws);
// Morton keys of sorted-state particles: key32 = m30, or key64 = m30<<32 | id
void jt_launch_morton(const float4* pos, const int* id, int64_t n, float box_half,
                      uint32_t* key32, uint64_t* key64, uint32_t* vals, cudaStream_t st);
// Stable LSD onesweep sort of (key, val) in place (keys/vals ping-pong through
// ws); shifts = bit offsets of the 8-bit digits, low to high.
int jt_radix_sort_u64(uint64_t* keys, uint32_t* vals, int64_t n, const int* shifts,
                      int npass, jt_sort_ws* ws, unsigned* d_err, cudaStream_t st);
// gather state by permutation: out[i] = in[perm[i]]
void jt_launch_reorder(const uint32_t* perm, int64_t n, const float4* pos_in,
                       float4* pos_out, const float4* vel_in, float4* vel_out,
                       const int* id_in, int* id_out, cudaStream_t st);
void jt_launch_split_keys(const uint64_t* key64, int64_t n, uint32_t* m30, uint32_t* tie,
                          cudaStream_t st);

// batched sort (jt_sort.cu): per-segment hist/status must be zeroed and the
// 4 tickets reset by the caller before the call
int jt_b_sort_reorder(const jt_seg_dev* d_segs, const jt_box_dev* d_boxes, int nseg,
                      const int64_t* d_pprefix, int64_t ntotal, const int64_t* d_tprefix,
                      int64_t ntiles, uint32_t* d_tickets, unsigned* d_err, cudaStream_t st);
int jt_sort_tile_size();

// tree (jt_tree.cu)
void jt_launch_karras(jt_tree_dev t, cudaStream_t st);
void jt_launch_moments_rc(jt_tree_dev t, const float4* pos, float mass, float box_half,
                          cudaStream_t st);

// batched tree build over segments (jt_tree.cu)
void jt_b_build_trees(const jt_seg_dev* d_segs, const jt_box_dev* d_boxes, int nseg,
                      const int64_t* d_iprefix, int64_t ninternal, const int64_t* d_pprefix,
                      int64_t nleaves, cudaStream_t st, const int* segflag = nullptr);

// RCOMPAT PM (jt_pm.cu): one CIC grid of the caller-order particles, the
// reference's Green's function in place, C2R to the potential.
struct jt_pm_dev {
    int M;
    double L;
    int order;               // 2 (CIC)
    int ngrid;               // 1
    float* rho;
    cufftComplex* force_k;   // potential spectrum
    float* force;            // potential grid
    cufftHandle plan_r2c, plan_c2r;
    int plans_ready;
};
void jt_launch_kspace_rc(cufftComplex* data, int M, double L, double r_s, int k_min, cudaStream_t st);
int jt_pm_tile_edge(int M);

// batched PM stages (jt_pm.cu)
void jt_b_tile_ranges(const jt_seg_dev* d_segs, const jt_box_dev* d_boxes, const int64_t* d_tprefix,
                      int nbox, int64_t ntiles, cudaStream_t st);
// src 0: the signed source D = sum s m W into B.rho; src 1: the unsigned
// source S = sum m W into B.rho_s (boxes without rho_s skip the pass).
// T: the largest tile edge of the pass; T16: every box's tile edge is 16.
int jt_b_deposit(const jt_seg_dev* d_segs, const jt_box_dev* d_boxes, const int64_t* d_tprefix,
                 int nbox, int64_t ntiles, int order, int ngrid, int T, cudaStream_t st, int src = 0,
                 bool T16 = false);
// The fused z transforms + k-space of 512^3 and 256^3 grids whose planes
// cuFFT transforms in 2D (jt_zfft.cu): CTAs per box (0 for other grid
// sizes), and the launches over every such box of a pass (sizes: bit 0 if
// the pass has 512^3 boxes, bit 1 if 256^3; src 1: a screened box's
// unsigned source).
int jt_zfft_tiles(int M);
int jt_b_zfft_kspace(const jt_box_dev* d_boxes, const int64_t* d_zprefix, int nbox, int64_t ntiles, int interlace,
                     int k_min, int src, int sizes, cudaStream_t st);
void jt_b_kspace(const jt_box_dev* d_boxes, const int64_t* d_kprefix, int nbox, int64_t nmodes,
                 int interlace, int k_min, cudaStream_t st);
// PM interpolation of every particle of the pass from each interlaced grid
// (tiles staged in shared memory): pmacc[b * npart + i], i = pprefix[seg] +
// index, the force of grid b on a unit m+ particle.  T: the largest tile edge
// of the pass (every box's T <= it; region (T + 4)^3 x 3 floats).
int jt_b_interp(const jt_seg_dev* d_segs, const jt_box_dev* d_boxes, const int64_t* d_tprefix,
                const int64_t* d_pprefix, int nbox, int64_t ntiles, int order, int ngrid, int T,
                int64_t npart, float4* pmacc, cudaStream_t st, bool T16 = false);

// walk (jt_walk.cu)
struct jt_walk_params {
    float L, halfL;
    float theta2;
    float rc2, rc;
    float eps2;
    float c;            // 1 / (2 r_s)
    float c2;           // c^2: the pair table's y = (r^2 + eps^2) c^2
    float slack;        // candidate prefilter: padding of the group's box
    float rc2_keep;     // candidate prefilter: widened cut
    float mass[2];      // per-species particle mass (G folded in) times c^3
    int M;
    float h_inv;        // M / L
    int order;          // PM assignment order (2 CIC, 3 TSC)
    int ngrid;          // PM grids (2 with interlacing)
    int parts;          // JT_PART_* bits: 1 = PM, 2 = tree
};
// Batched accurate walk over every segment's 32-particle groups (gprefix);
// every segment's tree arrays lie inside the arrays of `pool` (node arrays at
// a per-segment node offset, range at its particle offset, both < 2^31);
// stats[0] pair interactions inside r_cut, [1] node (multipole) interactions,
// [2] candidate particles distance-tested
int jt_b_walk(const jt_seg_dev* d_segs, const jt_box_dev* d_boxes, const int64_t* d_gprefix, int nseg,
              int64_t ngroups, const jt_tree_dev& pool, int order, int ngrid, int parts,
              float kick_frac, unsigned long long* stats, unsigned* d_err, cudaStream_t st,
              const int64_t* d_pprefix = nullptr, const unsigned char* tflag = nullptr,
              bool screened = false, const int* segflag = nullptr, const float4* pmacc = nullptr,
              int64_t npart = 0);
// Near-field cell list of a pass (cells of side >= r_cut, both species) and
// the cell walk over it: particles of cells whose 27-cell neighbourhood holds
// more than JT_CELL_KMAX candidates, and of boxes without a cell grid, are
// flagged in tflag for the tree walk; the others get their acceleration (and
// fused kick) here.  Scratch: ccount/cstart C + 1 ints, bsum, ccell/cslot,
// cpos/cid one entry per particle.
struct jt_cell_bufs {
    int* ccount; int* cstart; int* bsum; int* ccell; unsigned* cslot;
    float4* cpos; int2* cid; unsigned char* tflag;
    int* segflag;                 // per segment: some particle is flagged (its tree is built)
};
int jt_b_cells(const jt_seg_dev* d_segs, const jt_box_dev* d_boxes, const int64_t* d_pprefix, int nseg,
               int64_t npart, const int64_t* d_cprefix, int nbox, int64_t ncells, const jt_cell_bufs& cb,
               int order, int ngrid, int parts, float kick_frac, unsigned long long* stats,
               unsigned* d_err, cudaStream_t st, cudaEvent_t ev_walk0, cudaEvent_t ev_walk1,
               bool screened = false, const float4* pmacc = nullptr, bool count_pairs = true);
int jt_cell_scan_blocks(int64_t ncells);
// The cell counts per axis the batches' first force-only passes timed
// (jt_batch.cu), as text for jt_walk_tuning: "cells <n> particles: <default>
// -> <nb> per axis; ".
std::string jt_cell_tuning_text();
// Yukawa split factor S_Y(y) on the walk's table grid (y = (r_p / 2 r_s)^2
// over [0, 16], JT_STAB_N (value, next - value) entries) for b = kappa r_s.
// A pass with a screened box (jt_box_dev.ytab) runs the walks' screened
// instantiations (screened = true).
// The walks' pair-force table: G(y) = S(sqrt y) / y^{3/2} over
// y = (r_p / 2 r_s)^2 in [2^-32, 2^6), piecewise linear on 512 segments per
// octave (entry (a, b): G ~ a + b y), indexed by the float bits of y:
// entry = (bits(y) >> 14) - JT_LTAB_BASE, clamped to the last entry (zero).
// The pair force is then s_i s_j m_j c^3 G(y) d with c = 1 / (2 r_s): one
// table load and one FMA in place of a reciprocal square root and the split
// factor.  A screened box keeps the same table of the Yukawa kernel (S_Y in
// place of S, b = kappa r_s) for its opposite-species pairs.
constexpr int JT_LTAB_N = 38 * 512;
constexpr unsigned JT_LTAB_BASE = (127u - 32u) * 512u;
void jt_yukawa_log_table(double b, float2* tab);

// kick v += (a - drag v) kfrac*dt then drift x += v dfrac*dt, and the drift
// alone, with each box's own dt and drag (jt_box_dev)
void jt_b_kick_drift(const jt_seg_dev* d_segs, const jt_box_dev* d_boxes, const int64_t* d_prefix, int nseg,
                     int64_t ntotal, float kfrac, float dfrac, cudaStream_t st);
void jt_b_drift(const jt_seg_dev* d_segs, const jt_box_dev* d_boxes, const int64_t* d_prefix, int nseg,
                int64_t ntotal, float frac, cudaStream_t st);

struct jt_rc_params {
    float theta2, eps2, r_cut, box_half_q, r_s;   // quantised tree parameters
    float box_half, inv_cell, cell;               // PM (float) as the reference
    int M;
    float mass[2];
    int parts;                                    // JT_PART_* bits
    int screen;                                   // 1: Yukawa-screened full-range walk
    float inv_lambda;                             // quantised 1/lambda(z) (0 = off)
};
void jt_launch_walk_rcompat(const jt_rc_params& p, const float4* pos_caller,
                            const int8_t* sign_caller, int64_t n_all,
                            const float4* const spos[2], const int64_t n[2],
                            const jt_tree_dev tree[2], const float* phi,
                            float4* acc_caller, unsigned* d_err, cudaStream_t st);
void jt_launch_rcompat_deposit(const float4* pos_caller, const int8_t* sign_caller,
                               int64_t n_all, const float mass[2], float* rho, int M,
                               float box_half, float inv_cell, float inv_vol,
                               cudaStream_t st);

// step kernels (jt_walk.cu)
void jt_launch_kick(float4* vel, const float4* acc, int64_t n, float dt, float drag,
                    cudaStream_t st);
void jt_launch_drift(float4* pos, const float4* vel, int64_t n, float dt, float L,
                     float halfL, cudaStream_t st);
// caller-order gathers/scatters
void jt_launch_to_caller(const float4* src, const int* id, const int* gmap, int64_t n,
                         float4* dst, cudaStream_t st);
void jt_launch_aos_out(const float4* src, const int* id, const int* gmap, int64_t n,
                       float* dst_aos, cudaStream_t st);
void jt_launch_from_caller(const float4* src_caller, const int* id, const int* gmap, int64_t n,
                           float4* dst, cudaStream_t st);
void jt_launch_aos_in(const float* src_aos, int64_t n, float4* dst, int* id,
                      cudaStream_t st);
// Transfers through mapped pinned host memory (the host array's device
// address): every warp reads or writes whole contiguous 128-byte lines, staged
// through shared memory, so PCIe carries full lines.  host_in: dst[i] =
// src_aos[3i..3i+2] (and id[i] = i when id is given).  host_out: first
// jt_launch_inverse(id, n, inv) makes inv[id[i]] = i, then dst_aos[3k..3k+2] =
// src[inv[k]] in caller order k.
void jt_launch_host_in(const float* src_aos, int64_t n, float4* dst, int* id, cudaStream_t st);
void jt_launch_inverse(const int* id, int64_t n, int* inv, cudaStream_t st);
void jt_launch_host_out(const float4* src, const int* inv, int64_t n, float* dst_aos, cudaStream_t st);
void jt_launch_split_signed(const float* pos_aos, const float* vel_aos, const int8_t* sg,
                            int64_t n, const int* rank, float4* pos_p, float4* vel_p,
                            int* id_p, int* gmap_p, float4* pos_m, float4* vel_m,
                            int* id_m, int* gmap_m, cudaStream_t st);
