/*
 * CPU oracle for the bimetric TreePM force-and-step path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
 * calls this code.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline legs use it, and only as the checker / the timed CPU reference.
 *
 * Contents (each function cites the reference file:line it restates; paths
 * are relative to the janus-sim project root):
 *   ref_tree.c        GPU tree build of src/nbody_gpu_twopass.rs
 *                     (Morton keys, 64-bit key order, Karras nodes, leaves,
 *                     bottom-up COM/AABB reduce)            -- bit-exact
 *   ref_pm.c          GPU PM of src/nbody_gpu_twopass.rs + cuda/cufft_wrapper.cu
 *                     (CIC scatter, Green's function, FD gather)
 *   ref_walk.c        GPU erfc short-range walk of src/nbody_gpu_twopass.rs
 *                     with its warp-uniform (32-lane) decisions
 *   ref_cpu_treepm.c  CPU TreePM of src/treepm/{pm_grid,tree_short,
 *                     treepm_force}.rs (the reference CPU path; timed as the
 *                     CPU baseline)
 *   ewald.c           FP64 periodic direct-sum oracles (Ewald)
 *   acc_pm.c          FP64 PM in the accurate formulation (deconvolved,
 *                     spectral gradient) used to check the GPU PM kernels
 *   fft64.c           power-of-two complex FFT (f64), 1-D and 3-D
 */
#ifndef JANUS_ORACLE_H
#define JANUS_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- fft64.c ---------------- */
/* In-place complex FFT of length n (power of two); data interleaved re,im.
 * sign = -1 forward (exp(-i...)), +1 inverse; unnormalised. */
void orc_fft1d(double* data, int n, int sign);
/* 3-D in-place complex FFT of an M^3 array, index x + M*(y + M*z). */
void orc_fft3d(double* data, int M, int sign);

/* ---------------- ref_tree.c ---------------- */
uint32_t orc_expand10(uint32_t v);
void orc_morton30(const float* pos, int64_t n, float box_half, uint32_t* m30);
/* Order of the 64-bit keys (m30 << 32 | i): perm[k] = index of the k-th key. */
void orc_sort_keys(const uint32_t* m30, int64_t n, int32_t* perm);
/* Karras internal nodes over the sorted 64-bit keys (m30[perm[k]] << 32 | perm[k]).
 * Arrays sized 2n-1 (left/right/parent) and n-1 (rl/rr).  parent[0] = -1. */
void orc_karras(const uint32_t* m30_sorted, const int32_t* perm, int64_t n,
                int32_t* left, int32_t* right, int32_t* parent,
                int32_t* rl, int32_t* rr);
/* Leaves + bottom-up reduce.  pos_sorted: AoS xyz in sorted order.
 * node_pos: 7 floats/node (cx,cy,cz,hs,comx,comy,comz); node_mass; types. */
void orc_leaves_reduce(const float* pos_sorted, int64_t n, float box_half,
                       float mass_factor, const int32_t* left,
                       const int32_t* right, const int32_t* parent,
                       float* node_pos, float* node_mass, int32_t* types);
/* Full build: morton -> order -> gather -> karras -> leaves/reduce. */
void orc_build_tree(const float* pos, int64_t n, float box_half, float mass,
                    uint32_t* m30_sorted, int32_t* perm, float* pos_sorted,
                    int32_t* left, int32_t* right, int32_t* parent,
                    int32_t* rl, int32_t* rr,
                    float* node_pos, float* node_mass, int32_t* types);

/* ---------------- ref_pm.c ---------------- */
void orc_ref_cic_scatter(const float* pos, const int8_t* signs, int64_t n,
                         int M, float box_half, float inv_cell,
                         double* rho_plus, double* rho_minus);
void orc_ref_poisson(const double* rho, double* phi, int M, double box,
                     double g_constant, double r_s, int k_min);
void orc_ref_cic_gather(const float* pos, const int8_t* signs, int64_t n,
                        int M, float box_half, float inv_cell, float cell,
                        const double* phi_plus, const double* phi_minus,
                        float* pm_forces);
/* Whole reference PM force (scatter -> 2 solves -> gather), one mass factor. */
void orc_ref_pm_forces(const float* pos, const int8_t* signs, int64_t n,
                       int M, double box, double mass_factor, double r_cut,
                       int k_min, float* pm_forces);

/* ---------------- ref_walk.c ---------------- */
/* Host-side 16-bit parameter quantisation of the reference
 * (nbody_gpu_twopass.rs:1932-1937, 4079-4082 and kernel unpack 1684-1694). */
void orc_ref_quantize(double theta, double softening, double r_cut,
                      double box_size, float* theta_q, float* soft_q,
                      float* rcut_q, float* box_half_q);
void orc_ref_short_range(const float* pos_all, const int8_t* signs_all,
                         int64_t n_all, int tree_sign,
                         const float* node_pos, const float* node_mass,
                         const int32_t* left, const int32_t* right,
                         const int32_t* types,
                         float theta_q, float soft_q, float rcut_q,
                         float box_half_q, int accumulate, float* acc);
/* Complete reference force: PM + both trees (compute_short_range_forces). */
void orc_ref_total_forces(const float* pos_all, const int8_t* signs_all,
                          int64_t n_all, int M, double box, double theta,
                          double softening, double r_cut, double mass_factor,
                          int k_min, float* acc);

/* ---------------- ref_cpu_treepm.c ---------------- */
/* TreePMForce::new(r_cut, grid, box, theta, eps) + update + compute_all_forces
 * with per-particle masses (G folded in) and signs.  pos AoS f64.  Threads
 * from OpenMP (rayon in the reference). */
/* screened branch of compute_short_range_forces (ref_walk.c) */
void orc_ref_screen_quantize(double theta, double softening, double lambda_0, double z,
                             double box_size, float* theta_q, float* soft_q,
                             float* inv_lambda, float* box_half_q);
void orc_ref_screened_walk(const float* pos_all, const int8_t* signs_all,
                           int64_t n_all, int tree_sign,
                           const float* node_pos, const float* node_mass,
                           const int32_t* left, const int32_t* right,
                           const int32_t* types,
                           float theta, float softening, float inv_lambda,
                           float box_half, int accumulate, float* acc);
void orc_ref_total_forces_screened(const float* pos_all, const int8_t* signs_all,
                                   int64_t n_all, int M, double box, double theta,
                                   double softening, double r_cut, double mass_factor,
                                   int k_min, double lambda_0, double z, float* acc);

void orc_cpu_treepm_forces(const double* pos, const double* mass,
                           const int8_t* signs, int64_t n, double r_cut,
                           int grid, double box, double theta,
                           double softening, double* acc);
/* Timings of the last call (seconds): update (PM + tree build), forces. */
void orc_cpu_treepm_last_times(double* t_update, double* t_forces);

/* ---------------- ewald.c ---------------- */
/* Exact periodic split-model force on targets (FP64):
 *   long  = Ewald reciprocal sum with exp(-k^2 r_s^2) (no grid),
 *   short = sum over images of m r S(r_p)/r_p^3, r_p^2 = r^2 + eps^2,
 *           S(r) = erfc(r/2r_s) + (r/(r_s sqrt(pi))) exp(-r^2/4r_s^2),
 *           truncated at r_trunc (pass a large value for "no truncation").
 * With eps = 0 and r_trunc large this is the Ewald sum of 1/r^2 forces.
 * Sources: all n particles; targets: idx[0..nt).  signs +-1, masses >0. */
void orc_ewald_forces(const double* pos, const double* mass,
                      const int8_t* signs, int64_t n, const int64_t* idx,
                      int64_t nt, double box, double r_s, double eps,
                      double r_trunc, double kcut_tol, double* acc);
/* Long-range part only (reciprocal sum), same conventions. */
void orc_ewald_long(const double* pos, const double* mass, const int8_t* signs,
                    int64_t n, const int64_t* idx, int64_t nt, double box,
                    double r_s, double kcut_tol, double* acc);
/* Short-range part only (real-space, min image + images within r_trunc). */
void orc_ewald_short(const double* pos, const double* mass,
                     const int8_t* signs, int64_t n, const int64_t* idx,
                     int64_t nt, double box, double r_s, double eps,
                     double r_trunc, double* acc);

/* ---------------- acc_pm.c ---------------- */
/* FP64 PM in the accurate formulation: signed CIC deposit of s*m, Green
 * -4 pi/k^2 exp(-k^2 r_s^2) / W_cic(k)^2, spectral gradient (Nyquist
 * components of ik zeroed), CIC interpolation; acc = -s grad(phi). */
void orc_acc_pm_forces(const double* pos, const double* mass,
                       const int8_t* signs, int64_t n, int M, double box,
                       double r_s, int k_min, double* acc);
/* Same with assignment order (2 CIC, 3 TSC) and ngrid (1, or 2 interlaced). */
void orc_acc_pm_forces2(const double* pos, const double* mass,
                        const int8_t* signs, int64_t n, int M, double box,
                        double r_s, int k_min, int order, int ngrid, double* acc);
/* The three long-range force grids of the accurate formulation for the
 * signed source (acc of a + particle), index x + M*(y + M*z). */
void orc_acc_pm_grids(const double* pos, const double* mass,
                      const int8_t* signs, int64_t n, int M, double box,
                      double r_s, int k_min, double* fx, double* fy,
                      double* fz);

/* FP64 potential energy of the truncated split model (ewald.c) */
double orc_split_energy(const double* pos, const double* mass, const int8_t* signs, int64_t n,
                        double box, double r_s, double eps, double r_cut, double kcut_tol,
                        double* parts);

/* Yukawa-screened cross-species split model (ewald.c) */
void orc_ewald_forces_screened(const double* pos, const double* mass, const int8_t* signs, int64_t n,
                               const int64_t* idx, int64_t nt, double box, double r_s, double eps,
                               double r_trunc, double kappa, double kcut_tol, double* acc);

#ifdef __cplusplus
}
#endif
#endif
