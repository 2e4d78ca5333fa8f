/*
 * Restatement of the reference CPU TreePM.  TEST INFRASTRUCTURE ONLY
 * (the checker and the timed CPU baseline; never the product).
 *
 *   TreePMForce::new / update / compute_all_forces   src/treepm/treepm_force.rs:35-131
 *   PmGrid::assign_mass (f64 CIC, |m| weights, origin -L/2, rem_euclid)
 *                                                      src/treepm/pm_grid.rs:63-103
 *   PmGrid::solve_poisson_filtered (Green -4 pi G/k^2 exp(-k^2 r_s^2), k2 < 1e-10
 *                                   zeroed, 1/n^3)     src/treepm/pm_grid.rs:132-271
 *   PmGrid::interpolate_force (central differences /(2h) at the 8 CIC nodes,
 *                              F = -grad phi_same + grad phi_other)
 *                                                      src/treepm/pm_grid.rs:275-359
 *   TreePMTree::build_with_g (bounding box +-1 pad, cubic, 8-way octree, octant
 *                             by >= centre, per-species COM)
 *                                                      src/treepm/tree_short.rs:49-155
 *   acc_recursive / pairwise_acc_with_split (skip if r - 0.866 size >= r_cut;
 *       accept if size/r < theta and r < r_cut; pair weight 1-(r/r_cut)^4;
 *       no periodic images in the tree)                src/treepm/tree_short.rs:172-247
 *
 * Differences of form, not of result:
 *   - rustfft 6.4.1 (third-party, not vendored) is replaced by fft64.c, which
 *     computes the same unnormalised DFT; its lines run on OpenMP threads;
 *   - rayon's par_iter over targets becomes an OpenMP loop;
 *   - the octree is stored in flat arrays; children keep the reference's
 *     octant order and the per-node particle order (stable partition), so the
 *     COM sums run in the same order;
 *   - the reference recursion never ends for two particles at the same
 *     position; here a node deeper than 64 levels keeps its particles as a
 *     list of leaves (reached only by coincident points).
 * The reference passes mass per cell (not per volume) to the Green's function
 * with G = 1 (pm_grid.rs:99, treepm_force.rs:39); that scaling is kept.
 */
#include "oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <omp.h>

typedef struct {
    int32_t child[8];      /* -1 = empty; >=0 node index */
    int32_t leaf;          /* particle index if leaf, else -1 */
    int32_t first, count;  /* particle range in the ordered index array */
    double cx, cy, cz, size;
    double comp[3], mp, comm[3], mm;
} onode;

typedef struct {
    onode* nodes;
    int64_t n_nodes, cap;
    int64_t* order;  /* particle indices, grouped by node */
    int64_t* tmp;
} otree;

static int64_t new_node(otree* t)
{
    if (t->n_nodes == t->cap) {
        t->cap = t->cap ? 2 * t->cap : 1024;
        t->nodes = (onode*)realloc(t->nodes, sizeof(onode) * (size_t)t->cap);
    }
    memset(&t->nodes[t->n_nodes], 0, sizeof(onode));
    return t->n_nodes++;
}

static int64_t build_node(otree* t, const double* pos, const double* mass,
                          const int8_t* sg, int64_t first, int64_t count,
                          double minx, double miny, double minz,
                          double maxx, double maxy, double maxz, int depth)
{
    if (count == 0) return -1;
    int64_t id = new_node(t);
    onode* nd = &t->nodes[id];
    nd->first = (int32_t)first; nd->count = (int32_t)count;
    nd->cx = (minx + maxx) * 0.5; nd->cy = (miny + maxy) * 0.5; nd->cz = (minz + maxz) * 0.5;
    double dx = maxx - minx, dy = maxy - miny, dz = maxz - minz;
    nd->size = dx > dy ? dx : dy; nd->size = nd->size > dz ? nd->size : dz;
    for (int c = 0; c < 8; c++) nd->child[c] = -1;
    if (count == 1 || depth > 64) {
        nd->leaf = (int32_t)t->order[first];
        if (count > 1) nd->leaf = -2; /* coincident-point bucket */
        /* per-species COM of the bucket (used only for coincident points) */
        double sp[3] = {0, 0, 0}, mp = 0, sm[3] = {0, 0, 0}, mm = 0;
        for (int64_t q = first; q < first + count; q++) {
            int64_t i = t->order[q];
            if (sg[i] > 0) { sp[0] += pos[3*i] * mass[i]; sp[1] += pos[3*i+1] * mass[i]; sp[2] += pos[3*i+2] * mass[i]; mp += mass[i]; }
            else { sm[0] += pos[3*i] * mass[i]; sm[1] += pos[3*i+1] * mass[i]; sm[2] += pos[3*i+2] * mass[i]; mm += mass[i]; }
        }
        nd = &t->nodes[id];
        for (int d = 0; d < 3; d++) { nd->comp[d] = mp > 0 ? sp[d] / mp : 0; nd->comm[d] = mm > 0 ? sm[d] / mm : 0; }
        nd->mp = mp; nd->mm = mm;
        return id;
    }
    nd->leaf = -1;
    double cx = nd->cx, cy = nd->cy, cz = nd->cz;
    /* per-species COM over the node's particles in ascending index order
     * (tree_short.rs:113-140); the stable partition below keeps every node's
     * range ascending until its own children are built */
    double sp[3] = {0, 0, 0}, mp = 0, sm[3] = {0, 0, 0}, mm = 0;
    for (int64_t q = first; q < first + count; q++) {
        int64_t i = t->order[q];
        if (sg[i] > 0) {
            sp[0] += pos[3*i] * mass[i]; sp[1] += pos[3*i+1] * mass[i]; sp[2] += pos[3*i+2] * mass[i];
            mp += mass[i];
        } else {
            sm[0] += pos[3*i] * mass[i]; sm[1] += pos[3*i+1] * mass[i]; sm[2] += pos[3*i+2] * mass[i];
            mm += mass[i];
        }
    }
    /* stable 8-way partition by octant (tree_short.rs:98-104) */
    int64_t cnt[8] = {0}, off[8];
    for (int64_t q = first; q < first + count; q++) {
        int64_t i = t->order[q];
        int o = (pos[3*i] >= cx) | ((pos[3*i+1] >= cy) << 1) | ((pos[3*i+2] >= cz) << 2);
        cnt[o]++;
    }
    off[0] = first;
    for (int c = 1; c < 8; c++) off[c] = off[c - 1] + cnt[c - 1];
    int64_t w[8];
    for (int c = 0; c < 8; c++) w[c] = off[c];
    for (int64_t q = first; q < first + count; q++) {
        int64_t i = t->order[q];
        int o = (pos[3*i] >= cx) | ((pos[3*i+1] >= cy) << 1) | ((pos[3*i+2] >= cz) << 2);
        t->tmp[w[o]++] = i;
    }
    memcpy(t->order + first, t->tmp + first, sizeof(int64_t) * (size_t)count);
    int32_t ch[8];
    for (int c = 0; c < 8; c++) {
        /* BoundingBox::child_box (nbody.rs:150-163) */
        double bminx = (c & 1) ? cx : minx, bmaxx = (c & 1) ? maxx : cx;
        double bminy = (c & 2) ? cy : miny, bmaxy = (c & 2) ? maxy : cy;
        double bminz = (c & 4) ? cz : minz, bmaxz = (c & 4) ? maxz : cz;
        ch[c] = (int32_t)build_node(t, pos, mass, sg, off[c], cnt[c],
                                    bminx, bminy, bminz, bmaxx, bmaxy, bmaxz, depth + 1);
    }
    nd = &t->nodes[id];
    for (int c = 0; c < 8; c++) nd->child[c] = ch[c];
    if (mp > 0.0) { sp[0] /= mp; sp[1] /= mp; sp[2] /= mp; }
    if (mm > 0.0) { sm[0] /= mm; sm[1] /= mm; sm[2] /= mm; }
    for (int d = 0; d < 3; d++) { nd->comp[d] = sp[d]; nd->comm[d] = sm[d]; }
    nd->mp = mp; nd->mm = mm;
    return id;
}

/* pairwise_acc_with_split (tree_short.rs:219-247) */
static inline void pair_acc(const double* pi, int si, const double* pj, double mj,
                            int sj, double eps, double r_cut, double* a)
{
    if (mj == 0.0) return;
    double rx = pj[0] - pi[0], ry = pj[1] - pi[1], rz = pj[2] - pi[2];
    double r2 = rx * rx + ry * ry + rz * rz;
    double r = sqrt(r2);
    if (r >= r_cut) return;
    double r2s = r2 + eps * eps;
    if (r2s < 1e-20) return;
    double inter = (si == sj) ? 1.0 : -1.0;
    double inv = 1.0 / (r2s * sqrt(r2s));
    double s = inter * mj * inv;
    double x = r / r_cut, x2 = x * x;
    double wt = 1.0 - ((r >= r_cut) ? 1.0 : x2 * x2);
    a[0] += rx * s * wt; a[1] += ry * s * wt; a[2] += rz * s * wt;
}

static void acc_rec(const otree* t, int64_t id, const double* p, int s,
                    const double* pos, const double* mass, const int8_t* sg,
                    double eps, double theta, double r_cut, int64_t excl, double* a)
{
    if (id < 0) return;
    const onode* nd = &t->nodes[id];
    if (nd->leaf >= 0) {
        if (nd->leaf == excl) return;
        int64_t j = nd->leaf;
        pair_acc(p, s, pos + 3 * j, mass[j], sg[j] > 0 ? 1 : -1, eps, r_cut, a);
        return;
    }
    if (nd->leaf == -2) { /* coincident bucket: every member as a leaf */
        for (int64_t q = nd->first; q < nd->first + nd->count; q++) {
            int64_t j = t->order[q];
            if (j == excl) continue;
            pair_acc(p, s, pos + 3 * j, mass[j], sg[j] > 0 ? 1 : -1, eps, r_cut, a);
        }
        return;
    }
    double dx = p[0] - nd->cx, dy = p[1] - nd->cy, dz = p[2] - nd->cz;
    double r = sqrt(dx * dx + dy * dy + dz * dz);
    double size = nd->size;
    double mind = r - size * 0.866;
    if (mind < 0.0) mind = 0.0;
    if (mind >= r_cut) return;
    if (size / r < theta && r < r_cut) {
        pair_acc(p, s, nd->comp, nd->mp, 1, eps, r_cut, a);
        pair_acc(p, s, nd->comm, nd->mm, -1, eps, r_cut, a);
    } else {
        for (int c = 0; c < 8; c++)
            acc_rec(t, nd->child[c], p, s, pos, mass, sg, eps, theta, r_cut, excl, a);
    }
}

static double g_t_update, g_t_forces;

void orc_cpu_treepm_last_times(double* t_update, double* t_forces)
{
    *t_update = g_t_update; *t_forces = g_t_forces;
}

void orc_cpu_treepm_forces(const double* pos, const double* mass,
                           const int8_t* signs, int64_t n, double r_cut,
                           int M, double box, double theta,
                           double softening, double* acc)
{
    double t0 = omp_get_wtime();
    double r_s = r_cut / 3.0;
    double half = box / 2.0, gs = (double)M, h = box / M;
    int64_t G = (int64_t)M * M * M;
    /* --- PmGrid::clear + assign_mass (sequential, particle order) --- */
    double* rho[2];
    rho[0] = (double*)calloc((size_t)G, sizeof(double));
    rho[1] = (double*)calloc((size_t)G, sizeof(double));
    for (int64_t t = 0; t < n; t++) {
        double g[3]; int64_t ii[3]; double f[3];
        for (int d = 0; d < 3; d++) {
            g[d] = fmod((pos[3 * t + d] + half) / box * gs, gs);
            if (g[d] < 0) g[d] += gs;            /* rem_euclid */
            if (g[d] >= gs) g[d] -= gs;
            ii[d] = (int64_t)floor(g[d]);
            f[d] = g[d] - (double)ii[d];
        }
        double w[3][2] = {{1 - f[0], f[0]}, {1 - f[1], f[1]}, {1 - f[2], f[2]}};
        double* grid = signs[t] > 0 ? rho[0] : rho[1];
        double m = fabs(mass[t]);
        for (int di = 0; di < 2; di++)
            for (int dj = 0; dj < 2; dj++)
                for (int dk = 0; dk < 2; dk++) {
                    int64_t ci = (ii[0] + di) % M, cj = (ii[1] + dj) % M, ck = (ii[2] + dk) % M;
                    grid[ci + M * (cj + M * ck)] += m * (w[0][di] * w[1][dj] * w[2][dk]);
                }
    }
    /* --- solve_poisson_with_splitting(G = 1, r_s) for both grids --- */
    double* phi[2];
    double dk = 2.0 * M_PI / box;
    for (int s = 0; s < 2; s++) {
        double* c = (double*)malloc(sizeof(double) * 2 * (size_t)G);
        for (int64_t i = 0; i < G; i++) { c[2 * i] = rho[s][i]; c[2 * i + 1] = 0.0; }
        orc_fft3d(c, M, -1);
#pragma omp parallel for schedule(static)
        for (int64_t idx = 0; idx < G; idx++) {
            int64_t i = idx % M, j = (idx / M) % M, k = idx / ((int64_t)M * M);
            double ki = i <= M / 2 ? (double)i : (double)i - M;
            double kj = j <= M / 2 ? (double)j : (double)j - M;
            double kk = k <= M / 2 ? (double)k : (double)k - M;
            double k2 = (ki * ki + kj * kj + kk * kk) * dk * dk;
            if (k2 < 1e-10) { c[2 * idx] = 0; c[2 * idx + 1] = 0; continue; }
            double green = -4.0 * M_PI * 1.0 / k2;
            green *= exp(-k2 * (r_s * r_s));
            c[2 * idx] *= green; c[2 * idx + 1] *= green;
        }
        orc_fft3d(c, M, +1);
        phi[s] = (double*)malloc(sizeof(double) * (size_t)G);
        double norm = 1.0 / (double)G;
        for (int64_t i = 0; i < G; i++) phi[s][i] = c[2 * i] * norm;
        free(c);
    }
    /* --- TreePMTree::build_with_g --- */
    double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
    for (int64_t t = 0; t < n; t++)
        for (int d = 0; d < 3; d++) {
            if (pos[3 * t + d] < mn[d]) mn[d] = pos[3 * t + d];
            if (pos[3 * t + d] > mx[d]) mx[d] = pos[3 * t + d];
        }
    for (int d = 0; d < 3; d++) { mn[d] -= 1.0; mx[d] += 1.0; }
    double size = mx[0] - mn[0];
    if (mx[1] - mn[1] > size) size = mx[1] - mn[1];
    if (mx[2] - mn[2] > size) size = mx[2] - mn[2];
    double ctr[3] = {(mn[0] + mx[0]) / 2, (mn[1] + mx[1]) / 2, (mn[2] + mx[2]) / 2};
    otree tr = {0};
    tr.order = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    tr.tmp = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    for (int64_t i = 0; i < n; i++) tr.order[i] = i;
    int64_t root = build_node(&tr, pos, mass, signs, 0, n,
                              ctr[0] - size / 2, ctr[1] - size / 2, ctr[2] - size / 2,
                              ctr[0] + size / 2, ctr[1] + size / 2, ctr[2] + size / 2, 0);
    double t1 = omp_get_wtime();
    /* --- compute_all_forces (rayon -> OpenMP) --- */
#pragma omp parallel for schedule(dynamic, 256)
    for (int64_t t = 0; t < n; t++) {
        int s = signs[t] > 0 ? 1 : -1;
        const double* pa = s > 0 ? phi[0] : phi[1];
        const double* pr = s > 0 ? phi[1] : phi[0];
        double g[3]; int64_t ii[3]; double f[3];
        for (int d = 0; d < 3; d++) {
            g[d] = fmod((pos[3 * t + d] + half) / box * gs, gs);
            if (g[d] < 0) g[d] += gs;
            if (g[d] >= gs) g[d] -= gs;
            ii[d] = (int64_t)floor(g[d]);
            f[d] = g[d] - (double)ii[d];
        }
        double w[3][2] = {{1 - f[0], f[0]}, {1 - f[1], f[1]}, {1 - f[2], f[2]}};
        double F[3] = {0, 0, 0};
        for (int di = 0; di < 2; di++)
            for (int dj = 0; dj < 2; dj++)
                for (int dk2 = 0; dk2 < 2; dk2++) {
                    int64_t ci = (ii[0] + di) % M, cj = (ii[1] + dj) % M, ck = (ii[2] + dk2) % M;
                    double wt = w[0][di] * w[1][dj] * w[2][dk2];
                    int64_t cip = (ci + 1) % M, cim = (ci + M - 1) % M;
                    int64_t cjp = (cj + 1) % M, cjm = (cj + M - 1) % M;
                    int64_t ckp = (ck + 1) % M, ckm = (ck + M - 1) % M;
#define IX(a, b, c) ((a) + M * ((b) + M * (c)))
                    double dax = (pa[IX(cip, cj, ck)] - pa[IX(cim, cj, ck)]) / (2.0 * h);
                    double day = (pa[IX(ci, cjp, ck)] - pa[IX(ci, cjm, ck)]) / (2.0 * h);
                    double daz = (pa[IX(ci, cj, ckp)] - pa[IX(ci, cj, ckm)]) / (2.0 * h);
                    double drx = (pr[IX(cip, cj, ck)] - pr[IX(cim, cj, ck)]) / (2.0 * h);
                    double dry = (pr[IX(ci, cjp, ck)] - pr[IX(ci, cjm, ck)]) / (2.0 * h);
                    double drz = (pr[IX(ci, cj, ckp)] - pr[IX(ci, cj, ckm)]) / (2.0 * h);
#undef IX
                    F[0] += wt * (-dax + drx); F[1] += wt * (-day + dry); F[2] += wt * (-daz + drz);
                }
        double a[3] = {0, 0, 0};
        acc_rec(&tr, root, pos + 3 * t, s, pos, mass, signs, softening, theta, r_cut, t, a);
        acc[3 * t] = F[0] + a[0]; acc[3 * t + 1] = F[1] + a[1]; acc[3 * t + 2] = F[2] + a[2];
    }
    double t2 = omp_get_wtime();
    g_t_update = t1 - t0; g_t_forces = t2 - t1;
    free(rho[0]); free(rho[1]); free(phi[0]); free(phi[1]);
    free(tr.nodes); free(tr.order); free(tr.tmp);
}
