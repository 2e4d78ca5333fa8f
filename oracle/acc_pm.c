/*
 * FP64 particle-mesh force in the accurate formulation.  TEST INFRASTRUCTURE ONLY.
 *
 * This is the checker for the GPU long-range kernels (signed CIC deposit,
 * fused k-space kernel, three inverse transforms, CIC interpolation).  It is
 * the reference GPU PM (cuda/cufft_wrapper.cu:148-208, src/nbody_gpu_twopass.rs
 * :98-257) with three documented changes:
 *   - one signed source rho = sum_j s_j m_j W(x - x_j) / h^3 instead of two
 *     count grids (the reference's F+ = -grad phi+ + grad phi- is the same
 *     linear combination);
 *   - the Green's function -4 pi / k^2 exp(-k^2 r_s^2) is divided by the CIC
 *     window W(k)^2, W(k) = prod_d sinc^2(k_d h / 2), to undo assignment and
 *     interpolation smoothing;
 *   - the gradient is spectral (-i k phi); the component of i k along an axis
 *     whose index is the Nyquist index M/2 is set to zero.
 * Grid nodes sit at x = -L/2 + i h (the reference's origin); index x+M(y+Mz).
 */
#include "oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

static void deposit(const double* pos, const double* mass, const int8_t* signs,
                    int64_t n, int M, double box, double* rho)
{
    double half = box / 2.0, h = box / M, inv_vol = 1.0 / (h * h * h);
    for (int64_t t = 0; t < n; t++) {
        int64_t ii[3]; double f[3];
        for (int d = 0; d < 3; d++) {
            double g = (pos[3 * t + d] + half) / h;
            double fl = floor(g);
            f[d] = g - fl;
            int64_t gi = (int64_t)fl % M; if (gi < 0) gi += M;
            ii[d] = gi;
        }
        double q = (double)signs[t] * mass[t] * inv_vol;
        for (int dz = 0; dz < 2; dz++)
            for (int dy = 0; dy < 2; dy++)
                for (int dx = 0; dx < 2; dx++) {
                    double w = (dx ? f[0] : 1 - f[0]) * (dy ? f[1] : 1 - f[1]) * (dz ? f[2] : 1 - f[2]);
                    int64_t ci = (ii[0] + dx) % M, cj = (ii[1] + dy) % M, ck = (ii[2] + dz) % M;
                    rho[ci + M * (cj + M * ck)] += q * w;
                }
    }
}

static inline double sinc(double u) { return fabs(u) < 1e-12 ? 1.0 : sin(u) / u; }

void orc_acc_pm_grids(const double* pos, const double* mass,
                      const int8_t* signs, int64_t n, int M, double box,
                      double r_s, int k_min, double* fx, double* fy,
                      double* fz)
{
    int64_t G = (int64_t)M * M * M;
    double h = box / M, dk = 2.0 * M_PI / box;
    double* rho = (double*)calloc((size_t)G, sizeof(double));
    deposit(pos, mass, signs, n, M, box, rho);
    double* c = (double*)malloc(sizeof(double) * 2 * (size_t)G);
    for (int64_t i = 0; i < G; i++) { c[2 * i] = rho[i]; c[2 * i + 1] = 0; }
    free(rho);
    orc_fft3d(c, M, -1);
    double* out[3] = {fx, fy, fz};
    double* g = (double*)malloc(sizeof(double) * 2 * (size_t)G);
    for (int comp = 0; comp < 3; comp++) {
#pragma omp parallel for schedule(static)
        for (int64_t idx = 0; idx < G; idx++) {
            int n3[3] = {(int)(idx % M), (int)((idx / M) % M), (int)(idx / ((int64_t)M * M))};
            int ki[3]; double k[3], kg[3];
            int kmax = 0;
            for (int d = 0; d < 3; d++) {
                ki[d] = n3[d] <= M / 2 ? n3[d] : n3[d] - M;
                k[d] = dk * ki[d];
                kg[d] = (n3[d] == M / 2) ? 0.0 : k[d];
                int a = ki[d] < 0 ? -ki[d] : ki[d];
                if (a > kmax) kmax = a;
            }
            double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
            if (k2 == 0.0 || kmax < k_min) { g[2 * idx] = 0; g[2 * idx + 1] = 0; continue; }
            double w = 1.0;
            for (int d = 0; d < 3; d++) { double s = sinc(0.5 * k[d] * h); w *= s * s; }
            double green = -4.0 * M_PI / k2 * exp(-k2 * r_s * r_s) / (w * w);
            /* a(k) = -i k_comp phi(k) */
            double pr = c[2 * idx] * green, pi = c[2 * idx + 1] * green;
            g[2 * idx] = kg[comp] * pi;     /* -i*(pr + i pi)*kc = kc*(pi - i pr) */
            g[2 * idx + 1] = -kg[comp] * pr;
        }
        orc_fft3d(g, M, +1);
        for (int64_t i = 0; i < G; i++) out[comp][i] = g[2 * i] / (double)G;
    }
    free(g); free(c);
}

void orc_acc_pm_forces(const double* pos, const double* mass,
                       const int8_t* signs, int64_t n, int M, double box,
                       double r_s, int k_min, double* acc)
{
    int64_t G = (int64_t)M * M * M;
    double* F[3];
    for (int d = 0; d < 3; d++) F[d] = (double*)malloc(sizeof(double) * (size_t)G);
    orc_acc_pm_grids(pos, mass, signs, n, M, box, r_s, k_min, F[0], F[1], F[2]);
    double half = box / 2.0, h = box / M;
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < n; t++) {
        int64_t ii[3]; double f[3];
        for (int d = 0; d < 3; d++) {
            double gg = (pos[3 * t + d] + half) / h;
            double fl = floor(gg);
            f[d] = gg - fl;
            int64_t gi = (int64_t)fl % M; if (gi < 0) gi += M;
            ii[d] = gi;
        }
        double a[3] = {0, 0, 0};
        for (int dz = 0; dz < 2; dz++)
            for (int dy = 0; dy < 2; dy++)
                for (int dx = 0; dx < 2; dx++) {
                    double w = (dx ? f[0] : 1 - f[0]) * (dy ? f[1] : 1 - f[1]) * (dz ? f[2] : 1 - f[2]);
                    int64_t ci = (ii[0] + dx) % M, cj = (ii[1] + dy) % M, ck = (ii[2] + dz) % M;
                    int64_t id = ci + M * (cj + M * ck);
                    for (int d = 0; d < 3; d++) a[d] += w * F[d][id];
                }
        double s = (double)signs[t];
        acc[3 * t] = s * a[0]; acc[3 * t + 1] = s * a[1]; acc[3 * t + 2] = s * a[2];
    }
    for (int d = 0; d < 3; d++) free(F[d]);
}
