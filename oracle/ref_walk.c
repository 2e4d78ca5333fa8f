/*
 * Restatement of the reference GPU short-range walk.  TEST INFRASTRUCTURE ONLY.
 *
 *   forces_treepm_short_range   src/nbody_gpu_twopass.rs:1670-1811
 *   compute_short_range_forces  src/nbody_gpu_twopass.rs:3961-4138
 *   pack_rcut_boxhalf           src/nbody_gpu_twopass.rs:1932-1937
 *   forces_twopass_warpcoherent_screening  src/nbody_gpu_twopass.rs:911-1035
 *   pack_lambda_boxhalf         src/nbody_gpu_twopass.rs:1921-1927
 *
 * The kernel runs one thread per particle of the whole (both-species) array
 * and makes every traversal decision uniform across its 32-lane warp:
 *   - lane 0 owns a 128-entry stack (pushes only while sp < 127);
 *   - a node is skipped when EVERY lane has r - hs > r_cut (r to the node's
 *     geometric centre, minimum image);
 *   - the node is used as a monopole only when EVERY lane accepts it
 *     (leaf, or 4 hs^2 < theta^2 r^2); otherwise the warp descends;
 *   - lanes past the end of the array take particle 0's position and vote,
 *     but do not accumulate.
 * This file runs the 32 lanes of each warp as arrays in lock-step, which gives
 * the same decisions.  Pair force: s_i s_t m erfc(r_p/(2 r_s)) / r_p^3 (r_p^2 =
 * d^2 + eps^2 to the COM) when erfc > 1e-6, with r_s = r_cut_int / 3.
 * Float operations follow the kernel's order (compile with -ffp-contract=off).
 */
#include "oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

void orc_ref_quantize(double theta, double softening, double r_cut,
                      double box_size, float* theta_q, float* soft_q,
                      float* rcut_q, float* box_half_q)
{
    /* host: (x*1000) as u32 .min(0xFFFF) for theta and softening (:4079-4081);
     * r_cut and box_half truncated to integers (:1932-1937).  Rust `as u32`
     * saturates negatives to 0. */
    double tq = theta * 1000.0, sq = softening * 1000.0;
    uint32_t ti = tq <= 0.0 ? 0u : (tq >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)tq);
    uint32_t si = sq <= 0.0 ? 0u : (sq >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)sq);
    if (ti > 0xFFFF) ti = 0xFFFF;
    if (si > 0xFFFF) si = 0xFFFF;
    double bh = box_size / 2.0;
    uint32_t ri = r_cut <= 0.0 ? 0u : (uint32_t)r_cut;
    uint32_t bi = bh <= 0.0 ? 0u : (uint32_t)bh;
    if (ri > 0xFFFF) ri = 0xFFFF;
    if (bi > 0xFFFF) bi = 0xFFFF;
    /* kernel unpack (:1684-1691) */
    *theta_q = (float)ti / 1000.0f;
    *soft_q = (float)si / 1000.0f;
    *rcut_q = (float)ri;
    *box_half_q = (float)bi;
}

static inline float min_image(float d, float box_half)
{
    if (d > box_half) d -= 2.0f * box_half;
    if (d < -box_half) d += 2.0f * box_half;
    return d;
}

void orc_ref_short_range(const float* pos_all, const int8_t* signs_all,
                         int64_t n_all, int tree_sign,
                         const float* node_pos, const float* node_mass,
                         const int32_t* left, const int32_t* right,
                         const int32_t* types,
                         float theta, float softening, float r_cut,
                         float box_half, int accumulate, float* acc)
{
    float r_s = r_cut / 3.0f;
    float eps2 = softening * softening;
    float theta2 = theta * theta;
    int64_t n_warps = (n_all + 31) / 32;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t w = 0; w < n_warps; w++) {
        float px[32], py[32], pz[32], sf[32], ax[32], ay[32], az[32];
        int valid[32];
        for (int l = 0; l < 32; l++) {
            int64_t tid = w * 32 + l;
            valid[l] = tid < n_all;
            int64_t st = valid[l] ? tid : 0;
            px[l] = pos_all[3 * st]; py[l] = pos_all[3 * st + 1]; pz[l] = pos_all[3 * st + 2];
            sf[l] = ((int)signs_all[st] == tree_sign) ? 1.0f : -1.0f;
            ax[l] = ay[l] = az[l] = 0.0f;
        }
        int stack[128];
        int sp = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            int node = stack[--sp];
            if (node < 0) continue;
            int nt = types[node];
            if (nt == 0) continue;
            const float* p = node_pos + 7 * (int64_t)node;
            float cx = p[0], cy = p[1], cz = p[2], hs = p[3];
            float comx = p[4], comy = p[5], comz = p[6];
            float m = node_mass[node];
            int all_beyond = 1, all_approx = 1;
            for (int l = 0; l < 32; l++) {
                float dx = min_image(cx - px[l], box_half);
                float dy = min_image(cy - py[l], box_half);
                float dz = min_image(cz - pz[l], box_half);
                float r2 = dx * dx + dy * dy + dz * dz + 1e-20f;
                float r = sqrtf(r2);
                float closest = r - hs;
                if (!(closest > r_cut)) all_beyond = 0;
                int approx = (nt == 1) || ((4.0f * hs * hs) < (theta2 * r2));
                if (!approx) all_approx = 0;
            }
            if (all_beyond) continue;
            if (all_approx) {
                for (int l = 0; l < 32; l++) {
                    if (!valid[l]) continue;
                    float ddx = min_image(comx - px[l], box_half);
                    float ddy = min_image(comy - py[l], box_half);
                    float ddz = min_image(comz - pz[l], box_half);
                    float rp2 = ddx * ddx + ddy * ddy + ddz * ddz + eps2;
                    float rp = sqrtf(rp2);
                    float arg = rp / (2.0f * r_s);
                    float ef = erfcf(arg);
                    if (ef > 1e-6f) {
                        float irp3 = 1.0f / (rp * rp2);
                        float f = sf[l] * m * irp3 * ef;
                        ax[l] += f * ddx; ay[l] += f * ddy; az[l] += f * ddz;
                    }
                }
            } else {
                int lc = left[node], rc = right[node];
                if (rc >= 0 && sp < 127) stack[sp++] = rc;
                if (lc >= 0 && sp < 127) stack[sp++] = lc;
            }
        }
        for (int l = 0; l < 32; l++) {
            if (!valid[l]) continue;
            int64_t tid = w * 32 + l;
            if (accumulate) {
                acc[3 * tid] += ax[l]; acc[3 * tid + 1] += ay[l]; acc[3 * tid + 2] += az[l];
            } else {
                acc[3 * tid] = ax[l]; acc[3 * tid + 1] = ay[l]; acc[3 * tid + 2] = az[l];
            }
        }
    }
}

/* The screened branch of compute_short_range_forces (:4006-4068), used when
 * lambda_0 > 0.01: theta and softening ROUNDED to 1e-3 before the saturating
 * cast (:4009-4011), lambda(z) = lambda_0 sqrt(1 + z) in f64 (:4015) packed
 * with box_half by pack_lambda_boxhalf (truncated, :1921-1927); the kernel
 * unpacks lambda = lambda_int / 10 (:933-936) and uses 1/lambda when
 * lambda > 0.01, else no screening (:952). */
void orc_ref_screen_quantize(double theta, double softening, double lambda_0, double z,
                             double box_size, float* theta_q, float* soft_q,
                             float* inv_lambda, float* box_half_q)
{
    double tr = round(theta * 1000.0), sr = round(softening * 1000.0);
    uint32_t ti = tr <= 0.0 ? 0u : (tr >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)tr);
    uint32_t si = sr <= 0.0 ? 0u : (sr >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)sr);
    if (ti > 0xFFFF) ti = 0xFFFF;
    if (si > 0xFFFF) si = 0xFFFF;
    double l10 = lambda_0 * sqrt(1.0 + z) * 10.0, bh = box_size / 2.0;
    uint32_t li = !(l10 > 0.0) ? 0u : (l10 >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)l10);
    uint32_t bi = bh <= 0.0 ? 0u : (bh >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)bh);
    if (li > 0xFFFF) li = 0xFFFF;
    if (bi > 0xFFFF) bi = 0xFFFF;
    *theta_q = (float)ti / 1000.0f;
    *soft_q = (float)si / 1000.0f;
    float lam = (float)li / 10.0f;
    *inv_lambda = lam > 0.01f ? 1.0f / lam : 0.0f;
    *box_half_q = (float)bi;
}

/* forces_twopass_warpcoherent_screening (:911-1035): the warp-uniform walk of
 * orc_ref_short_range without the r_cut prune, over the full range, with
 * pair force s_i s_t S m / r_p^3 (no erfc); S = exp(-x)(1 + x), x = r_p /
 * lambda, for opposite signs when 1/lambda > 0, else 1. */
void orc_ref_screened_walk(const float* pos_all, const int8_t* signs_all,
                           int64_t n_all, int tree_sign,
                           const float* node_pos, const float* node_mass,
                           const int32_t* left, const int32_t* right,
                           const int32_t* types,
                           float theta, float softening, float inv_lambda,
                           float box_half, int accumulate, float* acc)
{
    float eps2 = softening * softening;
    float theta2 = theta * theta;
    int64_t n_warps = (n_all + 31) / 32;
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t w = 0; w < n_warps; w++) {
        float px[32], py[32], pz[32], ax[32], ay[32], az[32];
        int valid[32], same[32];
        for (int l = 0; l < 32; l++) {
            int64_t tid = w * 32 + l;
            valid[l] = tid < n_all;
            int64_t st = valid[l] ? tid : 0;
            px[l] = pos_all[3 * st]; py[l] = pos_all[3 * st + 1]; pz[l] = pos_all[3 * st + 2];
            same[l] = (int)signs_all[st] == tree_sign;
            ax[l] = ay[l] = az[l] = 0.0f;
        }
        int stack[128];
        int sp = 0;
        stack[sp++] = 0;
        while (sp > 0) {
            int node = stack[--sp];
            if (node < 0) continue;
            int nt = types[node];
            if (nt == 0) continue;
            const float* p = node_pos + 7 * (int64_t)node;
            float cx = p[0], cy = p[1], cz = p[2], hs = p[3];
            float comx = p[4], comy = p[5], comz = p[6];
            float m = node_mass[node];
            int all_approx = 1;
            for (int l = 0; l < 32; l++) {
                float dx = min_image(cx - px[l], box_half);
                float dy = min_image(cy - py[l], box_half);
                float dz = min_image(cz - pz[l], box_half);
                float r2 = dx * dx + dy * dy + dz * dz + 1e-20f;
                int approx = (nt == 1) || ((4.0f * hs * hs) < (theta2 * r2));
                if (!approx) all_approx = 0;
            }
            if (all_approx) {
                for (int l = 0; l < 32; l++) {
                    if (!valid[l]) continue;
                    float ddx = min_image(comx - px[l], box_half);
                    float ddy = min_image(comy - py[l], box_half);
                    float ddz = min_image(comz - pz[l], box_half);
                    float rp2 = ddx * ddx + ddy * ddy + ddz * ddz + eps2;
                    float rp = sqrtf(rp2);
                    float irp3 = 1.0f / (rp2 * rp);
                    float scr = 1.0f;
                    if (!same[l] && inv_lambda > 0.0f) {
                        float x = rp * inv_lambda;
                        scr = expf(-x) * (1.0f + x);
                    }
                    float sf = same[l] ? 1.0f : -1.0f;
                    float f = sf * scr * m * irp3;
                    ax[l] += f * ddx; ay[l] += f * ddy; az[l] += f * ddz;
                }
            } else {
                int lc = left[node], rc = right[node];
                if (rc >= 0 && sp < 127) stack[sp++] = rc;
                if (lc >= 0 && sp < 127) stack[sp++] = lc;
            }
        }
        for (int l = 0; l < 32; l++) {
            if (!valid[l]) continue;
            int64_t tid = w * 32 + l;
            if (accumulate) {
                acc[3 * tid] += ax[l]; acc[3 * tid + 1] += ay[l]; acc[3 * tid + 2] += az[l];
            } else {
                acc[3 * tid] = ax[l]; acc[3 * tid + 1] = ay[l]; acc[3 * tid + 2] = az[l];
            }
        }
    }
}

/* compute_short_range_forces (:3961-4138) followed by add_pm_forces (:67-78),
 * with the species extracted in array order (one valid outcome of the
 * reference's atomic compaction, :266-285).  lambda_0 > 0.01 takes the
 * screened branch (:3998, :4006-4068); the PM part is unchanged by it. */
static void total_forces(const float* pos_all, const int8_t* signs_all,
                         int64_t n_all, int M, double box, double theta,
                         double softening, double r_cut, double mass_factor,
                         int k_min, double lambda_0, double z, float* acc)
{
    const int screened = lambda_0 > 0.01;
    float tq, sq, rq, bq, il = 0.0f;
    if (screened)
        orc_ref_screen_quantize(theta, softening, lambda_0, z, box, &tq, &sq, &il, &bq);
    else
        orc_ref_quantize(theta, softening, r_cut, box, &tq, &sq, &rq, &bq);
    float box_half = (float)(box / 2.0);
    float* pm = (float*)malloc(sizeof(float) * 3 * (size_t)(n_all > 0 ? n_all : 1));
    orc_ref_pm_forces(pos_all, signs_all, n_all, M, box, mass_factor, r_cut, k_min, pm);
    for (int pass = 0; pass < 2; pass++) {
        int sign = pass == 0 ? 1 : -1;
        int64_t ns = 0;
        for (int64_t i = 0; i < n_all; i++) ns += ((int)signs_all[i] == sign);
        if (ns == 0) {
            if (pass == 0) memset(acc, 0, sizeof(float) * 3 * (size_t)n_all);
            continue;
        }
        float* ps = (float*)malloc(sizeof(float) * 3 * (size_t)ns);
        int64_t k = 0;
        for (int64_t i = 0; i < n_all; i++)
            if ((int)signs_all[i] == sign) {
                ps[3 * k] = pos_all[3 * i]; ps[3 * k + 1] = pos_all[3 * i + 1]; ps[3 * k + 2] = pos_all[3 * i + 2];
                k++;
            }
        int64_t nn = 2 * ns - 1;
        uint32_t* m30s = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)ns);
        int32_t* perm = (int32_t*)malloc(sizeof(int32_t) * (size_t)ns);
        float* pss = (float*)malloc(sizeof(float) * 3 * (size_t)ns);
        int32_t* lft = (int32_t*)malloc(sizeof(int32_t) * (size_t)nn);
        int32_t* rgt = (int32_t*)malloc(sizeof(int32_t) * (size_t)nn);
        int32_t* par = (int32_t*)malloc(sizeof(int32_t) * (size_t)nn);
        int32_t* rl = (int32_t*)malloc(sizeof(int32_t) * (size_t)(ns > 1 ? ns - 1 : 1));
        int32_t* rr = (int32_t*)malloc(sizeof(int32_t) * (size_t)(ns > 1 ? ns - 1 : 1));
        float* np7 = (float*)malloc(sizeof(float) * 7 * (size_t)nn);
        float* nm = (float*)malloc(sizeof(float) * (size_t)nn);
        int32_t* ty = (int32_t*)malloc(sizeof(int32_t) * (size_t)nn);
        orc_build_tree(ps, ns, box_half, (float)mass_factor, m30s, perm, pss,
                       lft, rgt, par, rl, rr, np7, nm, ty);
        if (screened)
            orc_ref_screened_walk(pos_all, signs_all, n_all, sign, np7, nm, lft, rgt, ty,
                                  tq, sq, il, bq, pass == 1, acc);
        else
            orc_ref_short_range(pos_all, signs_all, n_all, sign, np7, nm, lft, rgt, ty,
                                tq, sq, rq, bq, pass == 1, acc);
        free(ps); free(m30s); free(perm); free(pss); free(lft); free(rgt); free(par);
        free(rl); free(rr); free(np7); free(nm); free(ty);
    }
    for (int64_t i = 0; i < 3 * n_all; i++) acc[i] += pm[i];
    free(pm);
}

void orc_ref_total_forces(const float* pos_all, const int8_t* signs_all,
                          int64_t n_all, int M, double box, double theta,
                          double softening, double r_cut, double mass_factor,
                          int k_min, float* acc)
{
    total_forces(pos_all, signs_all, n_all, M, box, theta, softening, r_cut, mass_factor, k_min,
                 0.0, 0.0, acc);
}

void orc_ref_total_forces_screened(const float* pos_all, const int8_t* signs_all,
                                   int64_t n_all, int M, double box, double theta,
                                   double softening, double r_cut, double mass_factor,
                                   int k_min, double lambda_0, double z, float* acc)
{
    total_forces(pos_all, signs_all, n_all, M, box, theta, softening, r_cut, mass_factor, k_min,
                 lambda_0, z, acc);
}
