/*
 * Restatement of the reference GPU LBVH build.  TEST INFRASTRUCTURE ONLY.
 *
 * Follows src/nbody_gpu_twopass.rs (janus-sim):
 *   compute_morton_f32      :291-326  10 bits/axis, key = (m30 << 32) | index
 *   radix sort (8x8 bits)   :1521-1658, driven at :2400-2434  (sorts the unique
 *                           64-bit keys; any correct sort gives the same order)
 *   clz64_tp/delta_tp/range_tp/split_tp/build_bvh_tp  :356-447
 *   init_leaves_tp          :450-482
 *   reduce_tp               :485-561
 *
 * Float arithmetic is written operation for operation in the kernels' order;
 * compile with -ffp-contract=off so that no multiply-add is fused.  The CUDA
 * float->unsigned conversion saturates (negative or NaN -> 0), which is what
 * f2u_sat_rz reproduces; a plain C cast of a negative float is undefined.
 */
#include "oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

static uint32_t f2u_sat_rz(float x)
{
    if (!(x > 0.0f)) return 0u;               /* NaN, negatives, -0 */
    if (x >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint32_t)x;                        /* truncation toward zero */
}

uint32_t orc_expand10(uint32_t v)
{
    /* bit i of v -> bit 3i (expand10_tp, :302-310) */
    uint32_t r = 0;
    for (int i = 0; i < 10; i++) r |= ((v >> i) & 1u) << (3 * i);
    return r;
}

void orc_morton30(const float* pos, int64_t n, float box_half, uint32_t* m30)
{
    float scale = 1024.0f / (2.0f * box_half);
    for (int64_t i = 0; i < n; i++) {
        float x = (pos[3 * i] + box_half) * scale;
        float y = (pos[3 * i + 1] + box_half) * scale;
        float z = (pos[3 * i + 2] + box_half) * scale;
        uint32_t ix = f2u_sat_rz(x); if (ix > 0x3FFu) ix = 0x3FFu;
        uint32_t iy = f2u_sat_rz(y); if (iy > 0x3FFu) iy = 0x3FFu;
        uint32_t iz = f2u_sat_rz(z); if (iz > 0x3FFu) iz = 0x3FFu;
        m30[i] = orc_expand10(ix) | (orc_expand10(iy) << 1) | (orc_expand10(iz) << 2);
    }
}

static int cmp_u64(const void* a, const void* b)
{
    uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return (x > y) - (x < y);
}

void orc_sort_keys(const uint32_t* m30, int64_t n, int32_t* perm)
{
    uint64_t* k = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(n > 0 ? n : 1));
    for (int64_t i = 0; i < n; i++) k[i] = ((uint64_t)m30[i] << 32) | (uint64_t)(uint32_t)i;
    qsort(k, (size_t)n, sizeof(uint64_t), cmp_u64);
    for (int64_t i = 0; i < n; i++) perm[i] = (int32_t)(k[i] & 0xFFFFFFFFu);
    free(k);
}

static int clz64(uint64_t x) { return x ? __builtin_clzll(x) : 64; }

/* delta_tp (:369-373): common-prefix length of keys i and j, -1 outside. */
static int delta(const uint64_t* key, int64_t n, int64_t i, int64_t j)
{
    if (j < 0 || j >= n) return -1;
    if (key[i] == key[j]) return 64 + clz64((uint64_t)(uint32_t)((int32_t)i ^ (int32_t)j));
    return clz64(key[i] ^ key[j]);
}

void orc_karras(const uint32_t* m30_sorted, const int32_t* perm, int64_t n,
                int32_t* left, int32_t* right, int32_t* parent,
                int32_t* rl, int32_t* rr)
{
    if (n <= 0) return;
    int64_t n_nodes = 2 * n - 1;
    uint64_t* key = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
    for (int64_t i = 0; i < n; i++)
        key[i] = ((uint64_t)m30_sorted[i] << 32) | (uint64_t)(uint32_t)perm[i];
    for (int64_t i = 0; i < n_nodes; i++) { parent[i] = -1; left[i] = 0; right[i] = 0; }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n - 1; i++) {
        int64_t first, last;
        /* range_tp (:375-391) */
        if (i == 0) { first = 0; last = n - 1; }
        else {
            int dl = delta(key, n, i, i - 1);
            int dr = delta(key, n, i, i + 1);
            int d = (dr > dl) ? 1 : -1;
            int dmin = (d > 0) ? dl : dr;
            int64_t lmax = 2;
            while (delta(key, n, i, i + lmax * d) > dmin) lmax *= 2;
            int64_t l = 0;
            for (int64_t t = lmax / 2; t >= 1; t /= 2)
                if (delta(key, n, i, i + (l + t) * d) > dmin) l += t;
            int64_t j = i + l * d;
            if (d > 0) { first = i; last = j; } else { first = j; last = i; }
        }
        /* split_tp (:393-402) */
        int64_t gamma;
        if (first == last) gamma = first;
        else {
            int dn = delta(key, n, first, last);
            int64_t s = 0, t = last - first;
            while (t > 1) {
                t = (t + 1) / 2;
                if (delta(key, n, first, first + s + t) > dn) s += t;
            }
            gamma = first + s;
        }
        /* build_bvh_tp (:407-447): leaves are numbered n-1+j */
        int64_t lc = (first == gamma) ? (n - 1 + first) : gamma;
        int64_t rc = (gamma + 1 == last) ? (n - 1 + last) : (gamma + 1);
        left[i] = (int32_t)lc; right[i] = (int32_t)rc;
        rl[i] = (int32_t)first; rr[i] = (int32_t)last;
        parent[lc] = (int32_t)i; parent[rc] = (int32_t)i;
    }
    free(key);
}

void orc_leaves_reduce(const float* pos_sorted, int64_t n, float box_half,
                       float mass_factor, const int32_t* left,
                       const int32_t* right, const int32_t* parent,
                       float* node_pos, float* node_mass, int32_t* types)
{
    if (n <= 0) return;
    int64_t n_nodes = 2 * n - 1;
    int32_t* arrive = (int32_t*)calloc((size_t)n_nodes, sizeof(int32_t));
    for (int64_t i = 0; i < n_nodes; i++) { node_mass[i] = 0.0f; types[i] = 0; }
    float leaf_hs = box_half / 1024.0f;
    /* init_leaves_tp (:450-482) */
    for (int64_t i = 0; i < n; i++) {
        int64_t node = n - 1 + i;
        float* p = node_pos + 7 * node;
        float x = pos_sorted[3 * i], y = pos_sorted[3 * i + 1], z = pos_sorted[3 * i + 2];
        p[0] = x; p[1] = y; p[2] = z; p[3] = leaf_hs;
        p[4] = x; p[5] = y; p[6] = z;
        node_mass[node] = mass_factor;
        types[node] = 1;
    }
    /* reduce_tp (:485-561): the second child to arrive combines; the result
     * does not depend on arrival order, so threads run one after another. */
    for (int64_t leaf = 0; leaf < n; leaf++) {
        int64_t node = n - 1 + leaf;
        int64_t cur = parent[node];
        while (cur >= 0 && cur < n - 1) {
            int cnt = arrive[cur]++;
            if (cnt == 0) break;
            int64_t lc = left[cur], rc = right[cur];
            const float* L = node_pos + 7 * lc;
            const float* R = node_pos + 7 * rc;
            float* C = node_pos + 7 * cur;
            float ml = node_mass[lc], mr = node_mass[rc];
            float total = ml + mr;
            float com_x = (ml * L[4] + mr * R[4]) / total;
            float com_y = (ml * L[5] + mr * R[5]) / total;
            float com_z = (ml * L[6] + mr * R[6]) / total;
            float lcx = L[0], lcy = L[1], lcz = L[2], lhs = L[3];
            float rcx = R[0], rcy = R[1], rcz = R[2], rhs = R[3];
            float minx = fminf(lcx - lhs, rcx - rhs);
            float maxx = fmaxf(lcx + lhs, rcx + rhs);
            float miny = fminf(lcy - lhs, rcy - rhs);
            float maxy = fmaxf(lcy + lhs, rcy + rhs);
            float minz = fminf(lcz - lhs, rcz - rhs);
            float maxz = fmaxf(lcz + lhs, rcz + rhs);
            float cx = (minx + maxx) * 0.5f;
            float cy = (miny + maxy) * 0.5f;
            float cz = (minz + maxz) * 0.5f;
            float hs = fmaxf(fmaxf(maxx - minx, maxy - miny), maxz - minz) * 0.5f;
            if (hs < box_half / 1024.0f) hs = box_half / 1024.0f;
            C[0] = cx; C[1] = cy; C[2] = cz; C[3] = hs;
            C[4] = com_x; C[5] = com_y; C[6] = com_z;
            node_mass[cur] = total;
            types[cur] = 2;
            if (cur == 0) break;
            cur = parent[cur];
        }
    }
    free(arrive);
}

void orc_build_tree(const float* pos, int64_t n, float box_half, float mass,
                    uint32_t* m30_sorted, int32_t* perm, float* pos_sorted,
                    int32_t* left, int32_t* right, int32_t* parent,
                    int32_t* rl, int32_t* rr,
                    float* node_pos, float* node_mass, int32_t* types)
{
    if (n <= 0) return;
    uint32_t* m30 = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
    orc_morton30(pos, n, box_half, m30);
    orc_sort_keys(m30, n, perm);
    for (int64_t k = 0; k < n; k++) {
        int32_t s = perm[k];
        m30_sorted[k] = m30[s];
        pos_sorted[3 * k] = pos[3 * s];
        pos_sorted[3 * k + 1] = pos[3 * s + 1];
        pos_sorted[3 * k + 2] = pos[3 * s + 2];
    }
    orc_karras(m30_sorted, perm, n, left, right, parent, rl, rr);
    orc_leaves_reduce(pos_sorted, n, box_half, mass, left, right, parent,
                      node_pos, node_mass, types);
    free(m30);
}
