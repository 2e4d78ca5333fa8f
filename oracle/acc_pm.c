/*
 * FP64 particle-mesh force in the accurate formulation.  TEST INFRASTRUCTURE ONLY.
 *
 * This is the checker for the GPU long-range kernels (signed CIC deposit,
 * fused k-space kernel, three inverse transforms, CIC interpolation).  It is
 * the reference GPU PM (cuda/cufft_wrapper.cu:148-208, src/nbody_gpu_twopass.rs
 * :98-257) with these documented changes:
 *   - one signed source rho = sum_j s_j m_j W(x - x_j) / h^3 instead of two
 *     count grids (the reference's F+ = -grad phi+ + grad phi- is the same
 *     linear combination);
 *   - the Green's function -4 pi / k^2 exp(-k^2 r_s^2) is divided by the CIC
 *     window W(k)^2, W(k) = prod_d sinc^2(k_d h / 2), to undo assignment and
 *     interpolation smoothing;
 *   - the gradient is spectral (-i k phi); modes on a Nyquist plane are
 *     dropped (their weight is exp(-(pi r_s / h)^2), ~2e-7 at r_s = 1.25 h);
 *   - assignment of order 2 (CIC), 3 (TSC, deconvolved by sinc^6 per axis)
 *     or 4 (PCS, the cubic B-spline, sinc^8);
 *   - optional interlacing: a second grid with nodes half a cell higher on
 *     every axis, the spectra averaged with the phase of that shift, the
 *     force interpolated from both grids and averaged.
 * Grid nodes sit at x = -L/2 + i h (the reference's origin); index x+M(y+Mz).
 */
#include "oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdio.h>

/* stencil along one axis at grid coordinate g: first node and weights
 * (order 2 CIC: floor(g), +1; order 3 TSC: nearest node c, c-1..c+1;
 * order 4 PCS, the cubic B-spline: f = floor(g), nodes f-1..f+2) */
static int stencil(double g, int order, double* w)
{
    if (order == 2) {
        double f0 = floor(g), f = g - f0;
        w[0] = 1.0 - f; w[1] = f;
        return (int)f0;
    }
    if (order == 4) {
        double f0 = floor(g), t = g - f0, s = 1.0 - t;
        w[0] = s * s * s / 6.0;
        w[1] = 2.0 / 3.0 - t * t + 0.5 * t * t * t;
        w[2] = 2.0 / 3.0 - s * s + 0.5 * s * s * s;
        w[3] = t * t * t / 6.0;
        return (int)f0 - 1;
    }
    double c = floor(g + 0.5), d = g - c;
    w[0] = 0.5 * (0.5 - d) * (0.5 - d);
    w[1] = 0.75 - d * d;
    w[2] = 0.5 * (0.5 + d) * (0.5 + d);
    return (int)c - 1;
}

static void deposit(const double* pos, const double* mass, const int8_t* signs,
                    int64_t n, int M, double box, int order, double shift, double* rho)
{
    double half = box / 2.0, h = box / M, inv_vol = 1.0 / (h * h * h);
    for (int64_t t = 0; t < n; t++) {
        double w[3][4];
        int i0[3];
        for (int d = 0; d < 3; d++) i0[d] = stencil((pos[3 * t + d] + half) / h - shift, order, w[d]);
        double q = (double)signs[t] * mass[t] * inv_vol;
        for (int c = 0; c < order; c++)
            for (int b = 0; b < order; b++)
                for (int a = 0; a < order; a++) {
                    int64_t ci = ((i0[0] + a) % M + M) % M, cj = ((i0[1] + b) % M + M) % M,
                            ck = ((i0[2] + c) % M + M) % M;
                    rho[ci + M * (cj + M * ck)] += q * w[0][a] * w[1][b] * w[2][c];
                }
    }
}

static inline double sinc(double u) { return fabs(u) < 1e-12 ? 1.0 : sin(u) / u; }

/* force grids (3 per grid, ngrid = 1 or 2 interlaced) for an m+ particle */
void orc_acc_pm_grids2(const double* pos, const double* mass, const int8_t* signs, int64_t n,
                       int M, double box, double r_s, int k_min, int order, int ngrid,
                       double* F /* 3*ngrid*M^3 */)
{
    int64_t G = (int64_t)M * M * M;
    double h = box / M, dk = 2.0 * M_PI / box;
    double* c = (double*)calloc(2 * (size_t)G * ngrid, sizeof(double));
    double* rho = (double*)malloc(sizeof(double) * (size_t)G);
    for (int b = 0; b < ngrid; b++) {
        memset(rho, 0, sizeof(double) * (size_t)G);
        deposit(pos, mass, signs, n, M, box, order, 0.5 * b, rho);
        double* cb = c + 2 * (size_t)G * b;
        for (int64_t i = 0; i < G; i++) { cb[2 * i] = rho[i]; cb[2 * i + 1] = 0; }
        orc_fft3d(cb, M, -1);
    }
    free(rho);
    double* g = (double*)malloc(sizeof(double) * 2 * (size_t)G);
    for (int b = 0; b < ngrid; b++)
        for (int comp = 0; comp < 3; comp++) {
#pragma omp parallel for schedule(static)
            for (int64_t idx = 0; idx < G; idx++) {
                int n3[3] = {(int)(idx % M), (int)((idx / M) % M), (int)(idx / ((int64_t)M * M))};
                int ki[3], kmax = 0, nyq = 0;
                double k[3];
                for (int d = 0; d < 3; d++) {
                    ki[d] = n3[d] <= M / 2 ? n3[d] : n3[d] - M;
                    k[d] = dk * ki[d];
                    int a = ki[d] < 0 ? -ki[d] : ki[d];
                    if (a > kmax) kmax = a;
                    if (n3[d] == M / 2) nyq = 1;
                }
                double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
                if (k2 == 0.0 || kmax < k_min || nyq) { g[2 * idx] = 0; g[2 * idx + 1] = 0; continue; }
                double w = 1.0;
                for (int d = 0; d < 3; d++) w *= pow(sinc(0.5 * k[d] * h), 2.0 * order);
                double green = -4.0 * M_PI / k2 * exp(-k2 * r_s * r_s) / w;
                /* combined density: mean over grids of rho_b(k) exp(-i k.shift_b) */
                double rr = 0, ri = 0;
                for (int q = 0; q < ngrid; q++) {
                    double th = -0.5 * q * h * (k[0] + k[1] + k[2]);
                    double* cq = c + 2 * (size_t)G * q;
                    rr += cq[2 * idx] * cos(th) - cq[2 * idx + 1] * sin(th);
                    ri += cq[2 * idx] * sin(th) + cq[2 * idx + 1] * cos(th);
                }
                rr /= ngrid; ri /= ngrid;
                double pr = rr * green, pi = ri * green;
                double fr = k[comp] * pi, fi = -k[comp] * pr;   /* -i k phi */
                double th = 0.5 * b * h * (k[0] + k[1] + k[2]);  /* to the shifted nodes */
                g[2 * idx] = fr * cos(th) - fi * sin(th);
                g[2 * idx + 1] = fr * sin(th) + fi * cos(th);
            }
            orc_fft3d(g, M, +1);
            double* out = F + (size_t)G * (3 * b + comp);
            for (int64_t i = 0; i < G; i++) out[i] = g[2 * i] / (double)G;
        }
    free(g);
    free(c);
}

void orc_acc_pm_forces2(const double* pos, const double* mass, const int8_t* signs, int64_t n,
                        int M, double box, double r_s, int k_min, int order, int ngrid,
                        double* acc)
{
    int64_t G = (int64_t)M * M * M;
    double* F = (double*)malloc(sizeof(double) * 3 * (size_t)ngrid * (size_t)G);
    orc_acc_pm_grids2(pos, mass, signs, n, M, box, r_s, k_min, order, ngrid, F);
    double half = box / 2.0, h = box / M;
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < n; t++) {
        double a[3] = {0, 0, 0};
        for (int b = 0; b < ngrid; b++) {
            double w[3][4];
            int i0[3];
            for (int d = 0; d < 3; d++) i0[d] = stencil((pos[3 * t + d] + half) / h - 0.5 * b, order, w[d]);
            for (int c = 0; c < order; c++)
                for (int bb = 0; bb < order; bb++)
                    for (int aa = 0; aa < order; aa++) {
                        int64_t ci = ((i0[0] + aa) % M + M) % M, cj = ((i0[1] + bb) % M + M) % M,
                                ck = ((i0[2] + c) % M + M) % M;
                        int64_t id = ci + M * (cj + M * ck);
                        double wt = w[0][aa] * w[1][bb] * w[2][c];
                        for (int d = 0; d < 3; d++) a[d] += wt * F[(size_t)G * (3 * b + d) + id];
                    }
        }
        double s = (double)signs[t] / ngrid;
        acc[3 * t] = s * a[0]; acc[3 * t + 1] = s * a[1]; acc[3 * t + 2] = s * a[2];
    }
    free(F);
}

void orc_acc_pm_grids(const double* pos, const double* mass,
                      const int8_t* signs, int64_t n, int M, double box,
                      double r_s, int k_min, double* fx, double* fy,
                      double* fz)
{
    int64_t G = (int64_t)M * M * M;
    double* F = (double*)malloc(sizeof(double) * 3 * (size_t)G);
    orc_acc_pm_grids2(pos, mass, signs, n, M, box, r_s, k_min, 2, 1, F);
    memcpy(fx, F, sizeof(double) * (size_t)G);
    memcpy(fy, F + G, sizeof(double) * (size_t)G);
    memcpy(fz, F + 2 * G, sizeof(double) * (size_t)G);
    free(F);
}

void orc_acc_pm_forces(const double* pos, const double* mass,
                       const int8_t* signs, int64_t n, int M, double box,
                       double r_s, int k_min, double* acc)
{
    orc_acc_pm_forces2(pos, mass, signs, n, M, box, r_s, k_min, 2, 1, acc);
}
