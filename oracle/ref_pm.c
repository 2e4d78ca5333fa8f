/*
 * Restatement of the reference GPU particle-mesh path.  TEST INFRASTRUCTURE ONLY.
 *
 *   cic_scatter        src/nbody_gpu_twopass.rs:98-158   (count weights, f64 grids)
 *   cufft_solve_device cuda/cufft_wrapper.cu:350-398      (copy, D2Z, Green, Z2D, 1/N)
 *   apply_green_kernel cuda/cufft_wrapper.cu:148-208      (-4 pi G/k^2 exp(-k^2 r_s^2),
 *                                                         k_max < k_min and k=0 zeroed)
 *   cic_gather         src/nbody_gpu_twopass.rs:162-257  (central differences at the
 *                                                         8 CIC nodes; F = -grad phi_same
 *                                                         + grad phi_other)
 *   step_treepm_gpu    src/nbody_gpu_twopass.rs:4486-4600 (g_constant = mass_factor /
 *                                                         cell_vol, r_s = r_cut/3)
 *
 * The grid index is x + M*(y + M*z).  The reference's R2C halves the fastest
 * axis; the Green's function is symmetric in k, so a full complex transform
 * gives the same real potential.  Float operations follow the kernels' order
 * (compile with -ffp-contract=off).  Deposits are summed in particle order;
 * the GPU sums in atomic order, which differs only by f64 rounding.
 */
#include "oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

void orc_ref_cic_scatter(const float* pos, const int8_t* signs, int64_t n,
                         int M, float box_half, float inv_cell,
                         double* rho_plus, double* rho_minus)
{
    for (int64_t t = 0; t < n; t++) {
        float px = pos[3 * t], py = pos[3 * t + 1], pz = pos[3 * t + 2];
        float gx = (px + box_half) * inv_cell;
        float gy = (py + box_half) * inv_cell;
        float gz = (pz + box_half) * inv_cell;
        gx = fmodf(gx + (float)M, (float)M);
        gy = fmodf(gy + (float)M, (float)M);
        gz = fmodf(gz + (float)M, (float)M);
        int ix = (int)gx, iy = (int)gy, iz = (int)gz;
        float fx = gx - (float)ix, fy = gy - (float)iy, fz = gz - (float)iz;
        float wx[2] = {1.0f - fx, fx}, wy[2] = {1.0f - fy, fy}, wz[2] = {1.0f - fz, fz};
        double* grid = (signs[t] > 0) ? rho_plus : rho_minus;
        for (int di = 0; di < 2; di++)
            for (int dj = 0; dj < 2; dj++)
                for (int dk = 0; dk < 2; dk++) {
                    int ci = (ix + di) % M, cj = (iy + dj) % M, ck = (iz + dk) % M;
                    int64_t idx = ci + (int64_t)M * (cj + (int64_t)M * ck);
                    double w = (double)(wx[di] * wy[dj] * wz[dk]);
                    grid[idx] += w;
                }
    }
}

void orc_ref_poisson(const double* rho, double* phi, int M, double box,
                     double g_constant, double r_s, int k_min)
{
    int64_t G = (int64_t)M * M * M;
    double* c = (double*)malloc(sizeof(double) * 2 * (size_t)G);
    for (int64_t i = 0; i < G; i++) { c[2 * i] = rho[i]; c[2 * i + 1] = 0.0; }
    orc_fft3d(c, M, -1);
    double dk = 2.0 * 3.14159265358979323846 / box;
#pragma omp parallel for schedule(static)
    for (int64_t idx = 0; idx < G; idx++) {
        int kx = (int)(idx % M), ky = (int)((idx / M) % M), kz = (int)(idx / ((int64_t)M * M));
        int kxi = (kx <= M / 2) ? kx : kx - M;
        int kyi = (ky <= M / 2) ? ky : ky - M;
        int kzi = (kz <= M / 2) ? kz : kz - M;
        int ax = kxi < 0 ? -kxi : kxi, ay = kyi < 0 ? -kyi : kyi, az = kzi < 0 ? -kzi : kzi;
        int kmax = ax > ay ? ax : ay; kmax = kmax > az ? kmax : az;
        if (kmax < k_min) { c[2 * idx] = 0.0; c[2 * idx + 1] = 0.0; continue; }
        double kxv = kxi * dk, kyv = kyi * dk, kzv = kzi * dk;
        double k2 = kxv * kxv + kyv * kyv + kzv * kzv;
        if (k2 < 1e-20) { c[2 * idx] = 0.0; c[2 * idx + 1] = 0.0; continue; }
        double green = -4.0 * 3.14159265358979323846 * g_constant / k2;
        if (r_s > 0.0) green *= exp(-k2 * (r_s * r_s));
        c[2 * idx] *= green; c[2 * idx + 1] *= green;
    }
    orc_fft3d(c, M, +1);
    double factor = 1.0 / (double)G;
    for (int64_t i = 0; i < G; i++) phi[i] = c[2 * i] * factor;
    free(c);
}

void orc_ref_cic_gather(const float* pos, const int8_t* signs, int64_t n,
                        int M, float box_half, float inv_cell, float cell,
                        const double* phi_plus, const double* phi_minus,
                        float* pm_forces)
{
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < n; t++) {
        float px = pos[3 * t], py = pos[3 * t + 1], pz = pos[3 * t + 2];
        float gx = (px + box_half) * inv_cell;
        float gy = (py + box_half) * inv_cell;
        float gz = (pz + box_half) * inv_cell;
        gx = fmodf(gx + (float)M, (float)M);
        gy = fmodf(gy + (float)M, (float)M);
        gz = fmodf(gz + (float)M, (float)M);
        int ix = (int)gx, iy = (int)gy, iz = (int)gz;
        float fx = gx - (float)ix, fy = gy - (float)iy, fz = gz - (float)iz;
        float wx[2] = {1.0f - fx, fx}, wy[2] = {1.0f - fy, fy}, wz[2] = {1.0f - fz, fz};
        const double* pa = (signs[t] > 0) ? phi_plus : phi_minus;
        const double* pr = (signs[t] > 0) ? phi_minus : phi_plus;
        float fox = 0.0f, foy = 0.0f, foz = 0.0f;
        float h = cell;
        float inv_2h = 0.5f / h;
        for (int di = 0; di < 2; di++)
            for (int dj = 0; dj < 2; dj++)
                for (int dk = 0; dk < 2; dk++) {
                    int ci = (ix + di) % M, cj = (iy + dj) % M, ck = (iz + dk) % M;
                    float w = wx[di] * wy[dj] * wz[dk];
                    int cip = (ci + 1) % M, cim = (ci + M - 1) % M;
                    int cjp = (cj + 1) % M, cjm = (cj + M - 1) % M;
                    int ckp = (ck + 1) % M, ckm = (ck + M - 1) % M;
#define IDX(i, j, k) ((int64_t)(i) + (int64_t)M * ((int64_t)(j) + (int64_t)M * (int64_t)(k)))
                    float dax = (float)(pa[IDX(cip, cj, ck)] - pa[IDX(cim, cj, ck)]) * inv_2h;
                    float day = (float)(pa[IDX(ci, cjp, ck)] - pa[IDX(ci, cjm, ck)]) * inv_2h;
                    float daz = (float)(pa[IDX(ci, cj, ckp)] - pa[IDX(ci, cj, ckm)]) * inv_2h;
                    float drx = (float)(pr[IDX(cip, cj, ck)] - pr[IDX(cim, cj, ck)]) * inv_2h;
                    float dry = (float)(pr[IDX(ci, cjp, ck)] - pr[IDX(ci, cjm, ck)]) * inv_2h;
                    float drz = (float)(pr[IDX(ci, cj, ckp)] - pr[IDX(ci, cj, ckm)]) * inv_2h;
#undef IDX
                    fox += w * (-dax + drx);
                    foy += w * (-day + dry);
                    foz += w * (-daz + drz);
                }
        pm_forces[3 * t] = fox; pm_forces[3 * t + 1] = foy; pm_forces[3 * t + 2] = foz;
    }
}

void orc_ref_pm_forces(const float* pos, const int8_t* signs, int64_t n,
                       int M, double box, double mass_factor, double r_cut,
                       int k_min, float* pm_forces)
{
    int64_t G = (int64_t)M * M * M;
    float box_half = (float)(box / 2.0);
    float cell = (float)(box / M);
    float inv_cell = (float)(M / box);
    double cell_vol = pow(box / M, 3.0);
    double g_constant = mass_factor / cell_vol;
    double r_s = r_cut / 3.0;
    double* rp = (double*)calloc((size_t)G, sizeof(double));
    double* rm = (double*)calloc((size_t)G, sizeof(double));
    double* pp = (double*)malloc(sizeof(double) * (size_t)G);
    double* pmn = (double*)malloc(sizeof(double) * (size_t)G);
    orc_ref_cic_scatter(pos, signs, n, M, box_half, inv_cell, rp, rm);
    orc_ref_poisson(rp, pp, M, box, g_constant, r_s, k_min);
    orc_ref_poisson(rm, pmn, M, box, g_constant, r_s, k_min);
    orc_ref_cic_gather(pos, signs, n, M, box_half, inv_cell, cell, pp, pmn, pm_forces);
    free(rp); free(rm); free(pp); free(pmn);
}
