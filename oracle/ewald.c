/*
 * FP64 periodic direct-sum oracles.  TEST INFRASTRUCTURE ONLY.
 *
 * Janus pair rule (src/lib.rs:94-121): same signs attract, opposite signs
 * repel; acceleration of i = s_i * sum_j s_j m_j (x_j - x_i) / |r|^3 with G
 * folded into m.  The periodic sum is split the way the TreePM force is:
 *
 *   long:  a_L(i) = s_i sum_{k != 0} (4 pi / V) exp(-k^2 r_s^2) / k^2
 *                     * k * Im( exp(-i k.x_i) S(k) ),  S(k) = sum_j s_j m_j exp(i k.x_j)
 *          (Ewald reciprocal sum; the k-sum stops where exp(-k^2 r_s^2) < tol)
 *   short: a_S(i) = s_i sum_j sum_images s_j m_j r S(r_p) / r_p^3,
 *          r_p^2 = r^2 + eps^2,  S(r) = erfc(r/2r_s) + r/(r_s sqrt(pi)) exp(-r^2/4r_s^2)
 *          (pairs with |r| < r_trunc)
 *
 * With eps = 0 and r_trunc beyond the point where S vanishes this is the
 * Ewald sum of Newtonian forces, independent of r_s.  Pass r_trunc = r_cut
 * to evaluate the truncated TreePM split model exactly (no grid, no tree).
 *
 * Cost: the reciprocal sum is (number of k vectors) x (sources + targets);
 * exp(i k.x) is built from per-axis powers, so each k costs two complex
 * multiplies per particle.
 */
#include "oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

static inline double short_factor(double r, double r_s)
{
    double x = r / (2.0 * r_s);
    return erfc(x) + (r / (r_s * sqrt(M_PI))) * exp(-x * x);
}

void orc_ewald_short(const double* pos, const double* mass,
                     const int8_t* signs, int64_t n, const int64_t* idx,
                     int64_t nt, double box, double r_s, double eps,
                     double r_trunc, double* acc)
{
    /* cell list over sources with cells >= r_trunc when that gives >= 3 cells
     * per axis; otherwise loop over all sources and all images in range */
    int nc = (int)floor(box / r_trunc);
    double half = box / 2.0;
    int nimg = (int)ceil(r_trunc / box);  /* image shells needed */
    if (nc >= 3 && r_trunc <= half) {
        if (nc > 256) nc = 256;
        int64_t ncell = (int64_t)nc * nc * nc;
        int64_t* head = (int64_t*)malloc(sizeof(int64_t) * (size_t)ncell);
        int64_t* next = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
        for (int64_t c = 0; c < ncell; c++) head[c] = -1;
        double cs = box / nc;
        for (int64_t j = 0; j < n; j++) {
            int c[3];
            for (int d = 0; d < 3; d++) {
                double g = floor((pos[3 * j + d] + half) / cs);
                int gi = (int)g % nc; if (gi < 0) gi += nc;
                c[d] = gi;
            }
            int64_t cid = c[0] + (int64_t)nc * (c[1] + (int64_t)nc * c[2]);
            next[j] = head[cid]; head[cid] = j;
        }
#pragma omp parallel for schedule(dynamic, 64)
        for (int64_t q = 0; q < nt; q++) {
            int64_t i = idx[q];
            double a[3] = {0, 0, 0};
            int c[3];
            for (int d = 0; d < 3; d++) {
                double g = floor((pos[3 * i + d] + half) / cs);
                int gi = (int)g % nc; if (gi < 0) gi += nc;
                c[d] = gi;
            }
            for (int oz = -1; oz <= 1; oz++)
                for (int oy = -1; oy <= 1; oy++)
                    for (int ox = -1; ox <= 1; ox++) {
                        int cx = (c[0] + ox + nc) % nc, cy = (c[1] + oy + nc) % nc, cz = (c[2] + oz + nc) % nc;
                        for (int64_t j = head[cx + (int64_t)nc * (cy + (int64_t)nc * cz)]; j >= 0; j = next[j]) {
                            if (j == i) continue;
                            double r[3];
                            for (int d = 0; d < 3; d++) {
                                double dd = pos[3 * j + d] - pos[3 * i + d];
                                dd -= box * floor(dd / box + 0.5);
                                r[d] = dd;
                            }
                            double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
                            if (r2 >= r_trunc * r_trunc) continue;
                            double rp2 = r2 + eps * eps;
                            double rp = sqrt(rp2);
                            double f = (double)signs[j] * mass[j] * short_factor(rp, r_s) / (rp2 * rp);
                            a[0] += f * r[0]; a[1] += f * r[1]; a[2] += f * r[2];
                        }
                    }
            double s = (double)signs[i];
            acc[3 * q] = s * a[0]; acc[3 * q + 1] = s * a[1]; acc[3 * q + 2] = s * a[2];
        }
        free(head); free(next);
        return;
    }
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t q = 0; q < nt; q++) {
        int64_t i = idx[q];
        double a[3] = {0, 0, 0};
        for (int64_t j = 0; j < n; j++) {
            double r0[3];
            for (int d = 0; d < 3; d++) {
                double dd = pos[3 * j + d] - pos[3 * i + d];
                dd -= box * floor(dd / box + 0.5);
                r0[d] = dd;
            }
            for (int iz = -nimg; iz <= nimg; iz++)
                for (int iy = -nimg; iy <= nimg; iy++)
                    for (int ix = -nimg; ix <= nimg; ix++) {
                        if (j == i && ix == 0 && iy == 0 && iz == 0) continue;
                        double r[3] = {r0[0] + ix * box, r0[1] + iy * box, r0[2] + iz * box};
                        double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
                        if (r2 >= r_trunc * r_trunc) continue;
                        double rp2 = r2 + eps * eps;
                        double rp = sqrt(rp2);
                        double f = (double)signs[j] * mass[j] * short_factor(rp, r_s) / (rp2 * rp);
                        a[0] += f * r[0]; a[1] += f * r[1]; a[2] += f * r[2];
                    }
        }
        double s = (double)signs[i];
        acc[3 * q] = s * a[0]; acc[3 * q + 1] = s * a[1]; acc[3 * q + 2] = s * a[2];
    }
}

void orc_ewald_long(const double* pos, const double* mass, const int8_t* signs,
                    int64_t n, const int64_t* idx, int64_t nt, double box,
                    double r_s, double kcut_tol, double* acc)
{
    double dk = 2.0 * M_PI / box;
    double kmax = sqrt(-log(kcut_tol)) / r_s;   /* exp(-k^2 r_s^2) = tol */
    int nmax = (int)floor(kmax / dk);
    if (nmax < 1) nmax = 1;
    int W = nmax + 1;
    double V = box * box * box;
    /* list of half-space k vectors with weights 2 * (4 pi / V) e^{-k^2 r_s^2} / k^2 */
    int64_t cap = (int64_t)(2 * nmax + 1) * (2 * nmax + 1) * (nmax + 1);
    int* kv = (int*)malloc(sizeof(int) * 3 * (size_t)cap);
    double* kw = (double*)malloc(sizeof(double) * (size_t)cap);
    int64_t nk = 0;
    for (int nx = 0; nx <= nmax; nx++)
        for (int ny = -nmax; ny <= nmax; ny++)
            for (int nz = -nmax; nz <= nmax; nz++) {
                if (nx == 0 && (ny < 0 || (ny == 0 && nz <= 0))) continue;
                double k2 = dk * dk * (double)(nx * nx + ny * ny + nz * nz);
                if (k2 > kmax * kmax) continue;
                kv[3 * nk] = nx; kv[3 * nk + 1] = ny; kv[3 * nk + 2] = nz;
                kw[nk] = 2.0 * (4.0 * M_PI / V) * exp(-k2 * r_s * r_s) / k2;
                nk++;
            }
    /* per-particle axis powers e^{i n theta_d}, n = 0..nmax */
    int64_t np = n;
    double* ex = (double*)malloc(sizeof(double) * 2 * (size_t)W * 3 * (size_t)(np > 0 ? np : 1));
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < np; j++) {
        for (int d = 0; d < 3; d++) {
            double th = dk * pos[3 * j + d];
            double* e = ex + 2 * (size_t)W * (3 * j + d);
            for (int m = 0; m <= nmax; m++) { e[2 * m] = cos(m * th); e[2 * m + 1] = sin(m * th); }
        }
    }
    /* structure factors S(k) = sum_j s_j m_j e^{i k.x_j} */
    double* S = (double*)calloc(2 * (size_t)nk, sizeof(double));
#pragma omp parallel
    {
        double* Sl = (double*)calloc(2 * (size_t)nk, sizeof(double));
#pragma omp for schedule(static)
        for (int64_t j = 0; j < np; j++) {
            const double* e0 = ex + 2 * (size_t)W * (3 * j);
            const double* e1 = e0 + 2 * W;
            const double* e2 = e1 + 2 * W;
            double q = (double)signs[j] * mass[j];
            for (int64_t k = 0; k < nk; k++) {
                int a = kv[3 * k], b = kv[3 * k + 1], c = kv[3 * k + 2];
                double xr = e0[2 * a], xi = e0[2 * a + 1];
                double yr = e1[2 * (b < 0 ? -b : b)], yi = e1[2 * (b < 0 ? -b : b) + 1];
                if (b < 0) yi = -yi;
                double zr = e2[2 * (c < 0 ? -c : c)], zi = e2[2 * (c < 0 ? -c : c) + 1];
                if (c < 0) zi = -zi;
                double pr = xr * yr - xi * yi, pi = xr * yi + xi * yr;
                double er = pr * zr - pi * zi, ei = pr * zi + pi * zr;
                Sl[2 * k] += q * er; Sl[2 * k + 1] += q * ei;
            }
        }
#pragma omp critical
        for (int64_t k = 0; k < 2 * nk; k++) S[k] += Sl[k];
        free(Sl);
    }
#pragma omp parallel for schedule(static)
    for (int64_t t = 0; t < nt; t++) {
        int64_t i = idx[t];
        const double* e0 = ex + 2 * (size_t)W * (3 * i);
        const double* e1 = e0 + 2 * W;
        const double* e2 = e1 + 2 * W;
        double a0 = 0, a1 = 0, a2 = 0;
        for (int64_t k = 0; k < nk; k++) {
            int a = kv[3 * k], b = kv[3 * k + 1], c = kv[3 * k + 2];
            double xr = e0[2 * a], xi = e0[2 * a + 1];
            double yr = e1[2 * (b < 0 ? -b : b)], yi = e1[2 * (b < 0 ? -b : b) + 1];
            if (b < 0) yi = -yi;
            double zr = e2[2 * (c < 0 ? -c : c)], zi = e2[2 * (c < 0 ? -c : c) + 1];
            if (c < 0) zi = -zi;
            double pr = xr * yr - xi * yi, pi = xr * yi + xi * yr;
            double er = pr * zr - pi * zi, ei = pr * zi + pi * zr;
            /* Im(conj(E_i) S) */
            double im = er * S[2 * k + 1] - ei * S[2 * k];
            double f = kw[k] * im;
            a0 += f * (dk * a); a1 += f * (dk * b); a2 += f * (dk * c);
        }
        double s = (double)signs[i];
        acc[3 * t] = s * a0; acc[3 * t + 1] = s * a1; acc[3 * t + 2] = s * a2;
    }
    free(kv); free(kw); free(ex); free(S);
}

void orc_ewald_forces(const double* pos, const double* mass,
                      const int8_t* signs, int64_t n, const int64_t* idx,
                      int64_t nt, double box, double r_s, double eps,
                      double r_trunc, double kcut_tol, double* acc)
{
    double* al = (double*)malloc(sizeof(double) * 3 * (size_t)(nt > 0 ? nt : 1));
    orc_ewald_long(pos, mass, signs, n, idx, nt, box, r_s, kcut_tol, al);
    orc_ewald_short(pos, mass, signs, n, idx, nt, box, r_s, eps, r_trunc, acc);
    for (int64_t i = 0; i < 3 * nt; i++) acc[i] += al[i];
    free(al);
}

/*
 * Potential energy of the truncated split model (the force the engine
 * integrates), FP64, G folded into the masses, charges q = s m:
 *
 *   U = U_short + U_long + U_self
 *   U_short = -1/2 sum_{i != j, images} q_i q_j [psi(r_p) - psi(r_cp)]  for r < r_cut,
 *             psi(r) = erfc(r / 2r_s) / r, r_p^2 = r^2 + eps^2, r_cp^2 = r_cut^2 + eps^2
 *   U_long  = -(2 pi / V) sum_{k != 0} exp(-k^2 r_s^2) / k^2 |S(k)|^2
 *   U_self  = +(1 / (2 r_s sqrt(pi))) sum_i q_i^2
 *   U_bg    = +(2 pi r_s^2 / V) (sum_i q_i)^2  (the uniform background that
 *             the missing k = 0 mode stands for; constant in the positions,
 *             it makes U independent of r_s for a net charge)
 *
 * -grad_i U / m_i is the acceleration of orc_ewald_forces with r_trunc =
 * r_cut (the shift makes the short part continuous at r_cut, so U + KE is
 * conserved by the exact dynamics of the truncated model).  parts (may be
 * NULL) receives U_short, U_long, U_self + U_bg.
 */
double orc_split_energy(const double* pos, const double* mass, const int8_t* signs, int64_t n,
                        double box, double r_s, double eps, double r_cut, double kcut_tol,
                        double* parts)
{
    double half = box / 2.0;
    double rcp = sqrt(r_cut * r_cut + eps * eps);
    double psi_c = erfc(rcp / (2.0 * r_s)) / rcp;
    /* short: cell list with cells >= r_cut (falls back to all pairs) */
    int nc = (int)floor(box / r_cut);
    if (nc > 256) nc = 256;
    double us = 0.0;
    if (nc >= 3) {
        int64_t ncell = (int64_t)nc * nc * nc;
        int64_t* head = (int64_t*)malloc(sizeof(int64_t) * (size_t)ncell);
        int64_t* next = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
        for (int64_t c = 0; c < ncell; c++) head[c] = -1;
        double cs = box / nc;
        int* cell = (int*)malloc(sizeof(int) * 3 * (size_t)(n > 0 ? n : 1));
        for (int64_t j = 0; j < n; j++) {
            for (int d = 0; d < 3; d++) {
                int gi = (int)floor((pos[3 * j + d] + half) / cs) % nc;
                if (gi < 0) gi += nc;
                cell[3 * j + d] = gi;
            }
            int64_t cid = cell[3 * j] + (int64_t)nc * (cell[3 * j + 1] + (int64_t)nc * cell[3 * j + 2]);
            next[j] = head[cid];
            head[cid] = j;
        }
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : us)
        for (int64_t i = 0; i < n; i++) {
            double e = 0.0;
            for (int oz = -1; oz <= 1; oz++)
                for (int oy = -1; oy <= 1; oy++)
                    for (int ox = -1; ox <= 1; ox++) {
                        int cx = (cell[3 * i] + ox + nc) % nc, cy = (cell[3 * i + 1] + oy + nc) % nc,
                            cz = (cell[3 * i + 2] + oz + nc) % nc;
                        for (int64_t j = head[cx + (int64_t)nc * (cy + (int64_t)nc * cz)]; j >= 0; j = next[j]) {
                            if (j == i) continue;
                            double r2 = 0.0;
                            for (int d = 0; d < 3; d++) {
                                double dd = pos[3 * j + d] - pos[3 * i + d];
                                dd -= box * floor(dd / box + 0.5);
                                r2 += dd * dd;
                            }
                            if (r2 >= r_cut * r_cut) continue;
                            double rp = sqrt(r2 + eps * eps);
                            e += (double)signs[j] * mass[j] * (erfc(rp / (2.0 * r_s)) / rp - psi_c);
                        }
                    }
            us += -0.5 * (double)signs[i] * mass[i] * e;
        }
        free(head);
        free(next);
        free(cell);
    } else {
        int nimg = (int)ceil(r_cut / box);
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : us)
        for (int64_t i = 0; i < n; i++) {
            double e = 0.0;
            for (int64_t j = 0; j < n; j++)
                for (int iz = -nimg; iz <= nimg; iz++)
                    for (int iy = -nimg; iy <= nimg; iy++)
                        for (int ix = -nimg; ix <= nimg; ix++) {
                            if (j == i && ix == 0 && iy == 0 && iz == 0) continue;
                            double r2 = 0.0;
                            int sh[3] = {ix, iy, iz};
                            for (int d = 0; d < 3; d++) {
                                double dd = pos[3 * j + d] - pos[3 * i + d];
                                dd -= box * floor(dd / box + 0.5);
                                dd += sh[d] * box;
                                r2 += dd * dd;
                            }
                            if (r2 >= r_cut * r_cut) continue;
                            double rp = sqrt(r2 + eps * eps);
                            e += (double)signs[j] * mass[j] * (erfc(rp / (2.0 * r_s)) / rp - psi_c);
                        }
            us += -0.5 * (double)signs[i] * mass[i] * e;
        }
    }
    /* long: |S(k)|^2 over the half space of k (each pair k, -k once) */
    double dk = 2.0 * M_PI / box;
    double kmax = sqrt(-log(kcut_tol)) / r_s;
    int nmax = (int)floor(kmax / dk);
    if (nmax < 1) nmax = 1;
    double V = box * box * box;
    double ul = 0.0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : ul)
    for (int nx = 0; nx <= nmax; nx++) {
        double* cr = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
        double* ci = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
        for (int64_t j = 0; j < n; j++) {
            double th = dk * nx * pos[3 * j];
            cr[j] = cos(th);
            ci[j] = sin(th);
        }
        for (int ny = -nmax; ny <= nmax; ny++)
            for (int nz = -nmax; nz <= nmax; nz++) {
                if (nx == 0 && (ny < 0 || (ny == 0 && nz <= 0))) continue;
                double k2 = dk * dk * (double)(nx * nx + ny * ny + nz * nz);
                if (k2 > kmax * kmax) continue;
                double sr = 0.0, si = 0.0;
                for (int64_t j = 0; j < n; j++) {
                    double th = dk * (ny * pos[3 * j + 1] + nz * pos[3 * j + 2]);
                    double c = cos(th), s = sin(th);
                    double q = (double)signs[j] * mass[j];
                    sr += q * (cr[j] * c - ci[j] * s);
                    si += q * (cr[j] * s + ci[j] * c);
                }
                /* full-space (2 pi / V) sum = half-space (4 pi / V) sum */
                ul += -(4.0 * M_PI / V) * exp(-k2 * r_s * r_s) / k2 * (sr * sr + si * si);
            }
        free(cr);
        free(ci);
    }
    double q2 = 0.0, qt = 0.0;
    for (int64_t i = 0; i < n; i++) {
        q2 += mass[i] * mass[i];
        qt += (double)signs[i] * mass[i];
    }
    double uself = q2 / (2.0 * r_s * sqrt(M_PI)) + 2.0 * M_PI * r_s * r_s * qt * qt / V;
    if (parts) {
        parts[0] = us;
        parts[1] = ul;
        parts[2] = uself;
    }
    return us + ul + uself;
}

/*
 * Yukawa-screened cross-species force, FP64 split model.  Same-species pairs
 * are Newtonian, opposite-species pairs carry the screened potential
 * e^{-kappa r} / r (force e^{-kappa r}(1 + kappa r) / r^2, the reference's
 * screening factor, src/nbody_gpu_twopass.rs:1000-1017).  Split with
 * alpha = 1 / (2 r_s):
 *   Newton: short erfc(alpha r) / r,  long 4 pi e^{-k^2 r_s^2} / k^2;
 *   Yukawa: short (1 / 2r) [e^{-kr} erfc(alpha r - beta) + e^{kr} erfc(alpha r + beta)],
 *           beta = kappa r_s, long 4 pi e^{-(k^2 + kappa^2) r_s^2} / (k^2 + kappa^2)
 * (Ewald summation of the Yukawa potential).  The short-range force is the
 * derivative of the short potential at r_p (Plummer softening), cut at
 * r_trunc; the long part uses per-species structure factors.  kappa = 0 is
 * orc_ewald_forces.
 */
static double yukawa_short_force(double r, double r_s, double kappa)
{
    /* -d/dr of the short potential, times r^2 (the factor S of S m / r^2) */
    const double a = 1.0 / (2.0 * r_s), b = kappa * r_s;
    const double em = exp(-kappa * r), ep = exp(kappa * r);
    const double cm = erfc(a * r - b), cp = erfc(a * r + b);
    const double phi = 0.5 * (em * cm + ep * cp) / r;
    const double g = exp(-a * a * r * r - b * b);
    /* d/dr [e^{-kr} erfc(ar - b) + e^{kr} erfc(ar + b)] */
    const double dsum = -kappa * em * cm + kappa * ep * cp - 2.0 * (2.0 * a / sqrt(M_PI)) * g;
    const double dphi = -phi / r + 0.5 * dsum / r;
    return -dphi * r * r;
}

void orc_ewald_forces_screened(const double* pos, const double* mass, const int8_t* signs, int64_t n,
                               const int64_t* idx, int64_t nt, double box, double r_s, double eps,
                               double r_trunc, double kappa, double kcut_tol, double* acc)
{
    /* short part: all sources and the images within r_trunc */
    const int nimg = (int)ceil(r_trunc / box);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t q = 0; q < nt; q++) {
        const int64_t i = idx[q];
        double a[3] = {0, 0, 0};
        for (int64_t j = 0; j < n; j++) {
            double r0[3];
            for (int d = 0; d < 3; d++) {
                double dd = pos[3 * j + d] - pos[3 * i + d];
                dd -= box * floor(dd / box + 0.5);
                r0[d] = dd;
            }
            const int same = signs[j] == signs[i];
            for (int iz = -nimg; iz <= nimg; iz++)
                for (int iy = -nimg; iy <= nimg; iy++)
                    for (int ix = -nimg; ix <= nimg; ix++) {
                        if (j == i && ix == 0 && iy == 0 && iz == 0) continue;
                        const double r[3] = {r0[0] + ix * box, r0[1] + iy * box, r0[2] + iz * box};
                        const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
                        if (r2 >= r_trunc * r_trunc) continue;
                        const double rp2 = r2 + eps * eps, rp = sqrt(rp2);
                        const double S = same || kappa == 0.0 ? short_factor(rp, r_s)
                                                              : yukawa_short_force(rp, r_s, kappa);
                        const double f = (same ? 1.0 : -1.0) * mass[j] * S / (rp2 * rp);
                        a[0] += f * r[0]; a[1] += f * r[1]; a[2] += f * r[2];
                    }
        }
        acc[3 * q] = a[0]; acc[3 * q + 1] = a[1]; acc[3 * q + 2] = a[2];
    }
    /* long part: per-species structure factors S+(k), S-(k) (masses) */
    const double dk = 2.0 * M_PI / box, V = box * box * box;
    const double kmax = sqrt(-log(kcut_tol)) / r_s;
    int nmax = (int)floor(kmax / dk);
    if (nmax < 1) nmax = 1;
    double* al = (double*)calloc(3 * (size_t)(nt > 0 ? nt : 1), sizeof(double));
    for (int nx = 0; nx <= nmax; nx++)
        for (int ny = -nmax; ny <= nmax; ny++)
            for (int nz = -nmax; nz <= nmax; nz++) {
                if (nx == 0 && (ny < 0 || (ny == 0 && nz <= 0))) continue;
                const double k[3] = {dk * nx, dk * ny, dk * nz};
                const double k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
                if (k2 > kmax * kmax) continue;
                /* half space: each term twice */
                const double wN = 2.0 * (4.0 * M_PI / V) * exp(-k2 * r_s * r_s) / k2;
                const double wY = 2.0 * (4.0 * M_PI / V) * exp(-(k2 + kappa * kappa) * r_s * r_s) /
                                  (k2 + kappa * kappa);
                double sr[2] = {0, 0}, si[2] = {0, 0};
                for (int64_t j = 0; j < n; j++) {
                    const double th = k[0] * pos[3 * j] + k[1] * pos[3 * j + 1] + k[2] * pos[3 * j + 2];
                    const int s = signs[j] > 0 ? 0 : 1;
                    sr[s] += mass[j] * cos(th);
                    si[s] += mass[j] * sin(th);
                }
#pragma omp parallel for schedule(static)
                for (int64_t q = 0; q < nt; q++) {
                    const int64_t i = idx[q];
                    const double th = k[0] * pos[3 * i] + k[1] * pos[3 * i + 1] + k[2] * pos[3 * i + 2];
                    const double c = cos(th), sn = sin(th);
                    const int me = signs[i] > 0 ? 0 : 1, ot = 1 - me;
                    /* Im(e^{-ik.x_i} S(k)) for the same and the other species */
                    const double im_same = c * si[me] - sn * sr[me];
                    const double im_oth = c * si[ot] - sn * sr[ot];
                    const double f = wN * im_same - wY * im_oth;
                    al[3 * q] += f * k[0]; al[3 * q + 1] += f * k[1]; al[3 * q + 2] += f * k[2];
                }
            }
    for (int64_t q = 0; q < 3 * nt; q++) acc[q] += al[q];
    free(al);
}
