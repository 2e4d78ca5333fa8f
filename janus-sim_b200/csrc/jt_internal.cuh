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
    float t = __frcp_rn(fmaf(p, x, 1.0f));
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

// ---------------------------------------------------------------- launchers
// sort (jt_sort.cu)
int jt_sort_ws_alloc(jt_sort_ws* ws, int64_t cap, int max_passes);
void jt_sort_ws_free(jt_sort_ws* ws);
// Morton keys of sorted-state particles: key32 = m30, or key64 = m30<<32 | id
void jt_launch_morton(const float4* pos, const int* id, int64_t n, float box_half,
                      uint32_t* key32, uint64_t* key64, uint32_t* vals, cudaStream_t st);
// Stable LSD onesweep sort of (key, val) in place (keys/vals ping-pong through
// ws); shifts = bit offsets of the 8-bit digits, low to high.
int jt_radix_sort_u32(uint32_t* keys, uint32_t* vals, int64_t n, const int* shifts,
                      int npass, jt_sort_ws* ws, unsigned* d_err, cudaStream_t st);
int jt_radix_sort_u64(uint64_t* keys, uint32_t* vals, int64_t n, const int* shifts,
                      int npass, jt_sort_ws* ws, unsigned* d_err, cudaStream_t st);
// gather state by permutation: out[i] = in[perm[i]]
void jt_launch_reorder(const uint32_t* perm, int64_t n, const float4* pos_in,
                       float4* pos_out, const float4* vel_in, float4* vel_out,
                       const int* id_in, int* id_out, cudaStream_t st);
void jt_launch_split_keys(const uint64_t* key64, int64_t n, uint32_t* m30, uint32_t* tie,
                          cudaStream_t st);

// tree (jt_tree.cu)
void jt_launch_karras(jt_tree_dev t, cudaStream_t st);
void jt_launch_moments(jt_tree_dev t, const float4* pos, float mass, float box_half,
                       int rcompat, cudaStream_t st);

// PM (jt_pm.cu)
struct jt_pm_dev {
    int M;
    double L;
    int order;               // 2 = CIC, 3 = TSC (accurate); 2 in compatibility mode
    int ngrid;               // 1, or 2 with interlacing
    float* rho;              // ngrid grids
    cufftComplex* rho_k;     // ngrid spectra
    cufftComplex* force_k;   // 3*ngrid spectra + axis tables (ACCURATE) or 1 (RCOMPAT)
    float4* tabs;            // 2*M float4 axis tables (inside force_k)
    float* force;            // 3*ngrid grids (ACCURATE) or 1 potential grid (RCOMPAT)
    int4* ranges;            // per-tile particle ranges
    cufftHandle plan_r2c, plan_c2r;
    int plans_ready;
};
void jt_launch_deposit(const float4* pos0, int64_t n0, float q0, const float4* pos1,
                       int64_t n1, float q1, float* rho, int M, float L, int rcompat,
                       cudaStream_t st);
void jt_launch_kspace(const cufftComplex* rho_k, cufftComplex* out, int M, double L,
                      double r_s, int k_min, int rcompat, int interlace, const float4* tabs,
                      cudaStream_t st);
int jt_pm_tile_edge(int M);
// per-tile particle ranges [x,y) of species 0 and [z,w) of species 1
void jt_launch_tile_ranges(const uint32_t* m0, int64_t n0, const uint32_t* m1, int64_t n1,
                           int M, int4* ranges, cudaStream_t st);
int jt_launch_deposit_tiled(const float4* pos0, float q0, const float4* pos1, float q1,
                            const int4* ranges, float* rho, int M, float L, int order,
                            int ngrid, cudaStream_t st);

// walk (jt_walk.cu)
struct jt_walk_params {
    float L, halfL;
    float theta2;
    float rc2, rc;
    float eps2;
    float c;            // 1 / (2 r_s)
    float mass[2];      // per-species particle mass (G folded in)
    int M;
    float h_inv;        // M / L
    int order;          // PM assignment order (2 CIC, 3 TSC)
    int ngrid;          // PM grids (2 with interlacing)
    int parts;          // JT_PART_* bits: 1 = PM, 2 = tree
};
// stats[0] pair interactions inside r_cut, [1] node (multipole) interactions,
// [2] candidate particles distance-tested
void jt_launch_walk_accurate(const jt_walk_params& p, const float4* const pos[2],
                             const int64_t n[2], const jt_tree_dev tree[2],
                             const float* force3, float4* const acc[2],
                             float4* const vel[2], float kick_dt, float kick_drag,
                             unsigned long long* stats, unsigned* d_err, cudaStream_t st);

struct jt_rc_params {
    float theta2, eps2, r_cut, box_half_q, r_s;   // quantised tree parameters
    float box_half, inv_cell, cell;               // PM (float) as the reference
    int M;
    float mass[2];
    int parts;                                    // JT_PART_* bits
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
void jt_launch_split_signed(const float* pos_aos, const float* vel_aos, const int8_t* sg,
                            int64_t n, const int* rank, float4* pos_p, float4* vel_p,
                            int* id_p, int* gmap_p, float4* pos_m, float4* vel_m,
                            int* id_m, int* gmap_m, cudaStream_t st);
