// LBVH of one species: Karras internal nodes and bottom-up node moments.
//
// Numbering and child rules are the reference's (src/nbody_gpu_twopass.rs:
// 356-447, build_bvh_tp): internal nodes 0..n-2, leaf j at n-1+j; an internal
// node covers the key range [first, last] found from the common-prefix lengths
// delta(i, j) of the 64-bit keys (m30 << 32) | tie; its split gamma is found by
// the same halving search; the left child is leaf `first` when first == gamma,
// else internal node gamma; the right child is leaf `last` when gamma+1 ==
// last, else internal node gamma+1.  With tie = the caller's index this is the
// reference's key; the accurate path passes tie = sorted position (any unique,
// order-preserving tie gives a valid tree).
//
// Moments: one thread per leaf climbs towards the root; at each internal node
// the second child to arrive (atomic arrival counter) combines both children.
// Children's data is read through L2 (__ldcg) after the writer's
// __threadfence, so a stale L1 line is never used.
//   accurate : mass, centre of mass, tight AABB, second central moments
//              Q = sum m (x - com)(x - com)^T (parallel-axis combination)
//   rcompat  : the reference's reduce_tp (:485-561): COM = (ml*cl + mr*cr)/m
//              and the union of the children's cubes (leaf half-size
//              box_half/1024) as centre + half-size, floored at box_half/1024,
//              evaluated without fused multiply-adds so it matches the
//              reference operation for operation.
#include "jt_internal.cuh"

namespace {

__device__ __forceinline__ uint64_t tkey(const uint32_t* m30, const uint32_t* tie, int64_t i)
{
    uint32_t lo = tie ? tie[i] : (uint32_t)i;
    return ((uint64_t)m30[i] << 32) | lo;
}

__device__ __forceinline__ int tdelta(const uint32_t* m30, const uint32_t* tie, int64_t n,
                                      int64_t i, int64_t j)
{
    if (j < 0 || j >= n) return -1;
    uint64_t a = tkey(m30, tie, i), b = tkey(m30, tie, j);
    if (a == b) return 64 + __clzll((long long)(uint64_t)(uint32_t)((int32_t)i ^ (int32_t)j));
    return __clzll((long long)(a ^ b));
}

__global__ void k_karras(const uint32_t* __restrict__ m30, const uint32_t* __restrict__ tie,
                         int64_t n, int2* __restrict__ child, int* __restrict__ parent,
                         int2* __restrict__ range)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int64_t first, last;
    if (i == 0) {
        first = 0;
        last = n - 1;
    } else {
        int dl = tdelta(m30, tie, n, i, i - 1);
        int dr = tdelta(m30, tie, n, i, i + 1);
        int d = (dr > dl) ? 1 : -1;
        int dmin = (d > 0) ? dl : dr;
        int64_t lmax = 2;
        while (tdelta(m30, tie, n, i, i + lmax * d) > dmin) lmax *= 2;
        int64_t l = 0;
        for (int64_t t = lmax / 2; t >= 1; t /= 2)
            if (tdelta(m30, tie, n, i, i + (l + t) * d) > dmin) l += t;
        int64_t j = i + l * d;
        first = d > 0 ? i : j;
        last = d > 0 ? j : i;
    }
    int64_t gamma = first;
    if (first != last) {
        int dn = tdelta(m30, tie, n, first, last);
        int64_t s = 0, t = last - first;
        while (t > 1) {
            t = (t + 1) / 2;
            if (tdelta(m30, tie, n, first, first + s + t) > dn) s += t;
        }
        gamma = first + s;
    }
    int64_t lc = (first == gamma) ? (n - 1 + first) : gamma;
    int64_t rc = (gamma + 1 == last) ? (n - 1 + last) : (gamma + 1);
    child[i] = make_int2((int)lc, (int)rc);
    if (range) range[i] = make_int2((int)first, (int)last);
    parent[lc] = (int)i;
    parent[rc] = (int)i;
}

template <bool RC>
__global__ void k_moments(int64_t n, const float4* __restrict__ pos, float mass, float box_half,
                          const int2* __restrict__ child, const int* __restrict__ parent,
                          int* __restrict__ flag, float4* com, float4* bmin, float4* bmax,
                          float4* quad0, float2* quad1)
{
    int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    int64_t node = n - 1 + j;
    float4 p = pos[j];
    float leaf_hs = box_half / 1024.0f;
    com[node] = make_float4(p.x, p.y, p.z, mass);
    if (RC) {
        bmin[node] = make_float4(p.x, p.y, p.z, leaf_hs);
    } else {
        bmin[node] = make_float4(p.x, p.y, p.z, 0.0f);
        bmax[node] = make_float4(p.x, p.y, p.z, 0.0f);
        quad0[node] = make_float4(0.f, 0.f, 0.f, 0.f);
        quad1[node] = make_float2(0.f, 0.f);
    }
    int cur = parent[node];
    while (cur >= 0) {
        __threadfence();
        if (atomicAdd(&flag[cur], 1) == 0) return;  // first child: the sibling finishes
        int2 ch = __ldcg(&child[cur]);
        float4 cl = __ldcg(&com[ch.x]);
        float4 cr = __ldcg(&com[ch.y]);
        if (RC) {
            float ml = cl.w, mr = cr.w;
            float tot = __fadd_rn(ml, mr);
            float cx = __fdiv_rn(__fadd_rn(__fmul_rn(ml, cl.x), __fmul_rn(mr, cr.x)), tot);
            float cy = __fdiv_rn(__fadd_rn(__fmul_rn(ml, cl.y), __fmul_rn(mr, cr.y)), tot);
            float cz = __fdiv_rn(__fadd_rn(__fmul_rn(ml, cl.z), __fmul_rn(mr, cr.z)), tot);
            float4 bl = __ldcg(&bmin[ch.x]);
            float4 br = __ldcg(&bmin[ch.y]);
            float minx = fminf(__fsub_rn(bl.x, bl.w), __fsub_rn(br.x, br.w));
            float maxx = fmaxf(__fadd_rn(bl.x, bl.w), __fadd_rn(br.x, br.w));
            float miny = fminf(__fsub_rn(bl.y, bl.w), __fsub_rn(br.y, br.w));
            float maxy = fmaxf(__fadd_rn(bl.y, bl.w), __fadd_rn(br.y, br.w));
            float minz = fminf(__fsub_rn(bl.z, bl.w), __fsub_rn(br.z, br.w));
            float maxz = fmaxf(__fadd_rn(bl.z, bl.w), __fadd_rn(br.z, br.w));
            float ccx = __fmul_rn(__fadd_rn(minx, maxx), 0.5f);
            float ccy = __fmul_rn(__fadd_rn(miny, maxy), 0.5f);
            float ccz = __fmul_rn(__fadd_rn(minz, maxz), 0.5f);
            float hs = __fmul_rn(fmaxf(fmaxf(__fsub_rn(maxx, minx), __fsub_rn(maxy, miny)),
                                       __fsub_rn(maxz, minz)), 0.5f);
            if (hs < leaf_hs) hs = leaf_hs;
            com[cur] = make_float4(cx, cy, cz, tot);
            bmin[cur] = make_float4(ccx, ccy, ccz, hs);
        } else {
            float ml = cl.w, mr = cr.w, m = ml + mr;
            float inv = 1.0f / m;
            float cx = (ml * cl.x + mr * cr.x) * inv;
            float cy = (ml * cl.y + mr * cr.y) * inv;
            float cz = (ml * cl.z + mr * cr.z) * inv;
            float4 lo_l = __ldcg(&bmin[ch.x]), lo_r = __ldcg(&bmin[ch.y]);
            float4 hi_l = __ldcg(&bmax[ch.x]), hi_r = __ldcg(&bmax[ch.y]);
            float4 ql0 = __ldcg(&quad0[ch.x]), qr0 = __ldcg(&quad0[ch.y]);
            float2 ql1 = __ldcg(&quad1[ch.x]), qr1 = __ldcg(&quad1[ch.y]);
            float dlx = cl.x - cx, dly = cl.y - cy, dlz = cl.z - cz;
            float drx = cr.x - cx, dry = cr.y - cy, drz = cr.z - cz;
            float4 q0;
            q0.x = ql0.x + qr0.x + ml * dlx * dlx + mr * drx * drx;
            q0.y = ql0.y + qr0.y + ml * dly * dly + mr * dry * dry;
            q0.z = ql0.z + qr0.z + ml * dlz * dlz + mr * drz * drz;
            q0.w = ql0.w + qr0.w + ml * dlx * dly + mr * drx * dry;
            float2 q1;
            q1.x = ql1.x + qr1.x + ml * dlx * dlz + mr * drx * drz;
            q1.y = ql1.y + qr1.y + ml * dly * dlz + mr * dry * drz;
            com[cur] = make_float4(cx, cy, cz, m);
            bmin[cur] = make_float4(fminf(lo_l.x, lo_r.x), fminf(lo_l.y, lo_r.y),
                                    fminf(lo_l.z, lo_r.z), 0.0f);
            bmax[cur] = make_float4(fmaxf(hi_l.x, hi_r.x), fmaxf(hi_l.y, hi_r.y),
                                    fmaxf(hi_l.z, hi_r.z), 0.0f);
            quad0[cur] = q0;
            quad1[cur] = q1;
        }
        cur = parent[cur];
    }
}

}  // namespace

void jt_launch_karras(jt_tree_dev t, cudaStream_t st)
{
    if (t.n <= 0) return;
    int64_t nn = 2 * t.n - 1;
    cudaMemsetAsync(t.parent, 0xFF, sizeof(int) * nn, st);   // parent[root] = -1
    cudaMemsetAsync(t.child, 0, sizeof(int2) * nn, st);
    if (t.n >= 2)
        k_karras<<<(unsigned)((t.n - 1 + 255) / 256), 256, 0, st>>>(t.m30, t.tie, t.n, t.child,
                                                                   t.parent, t.range);
}

// RCOMPAT node moments (the accurate path builds its moments in k_b_moments)
void jt_launch_moments_rc(jt_tree_dev t, const float4* pos, float mass, float box_half, cudaStream_t st)
{
    if (t.n <= 0) return;
    cudaMemsetAsync(t.flag, 0, sizeof(int) * (t.n > 1 ? t.n - 1 : 1), st);
    unsigned g = (unsigned)((t.n + 255) / 256);
    k_moments<true><<<g, 256, 0, st>>>(t.n, pos, mass, box_half, t.child, t.parent, t.flag, t.com, t.bmin,
                                       t.bmax, t.quad0, t.quad1);
}

// ======================================================================
// Batched versions over segments (accurate mode: tie = sorted position).
// ======================================================================
namespace {

// internal nodes of every segment; iprefix counts n-1 per segment.  Node 0's
// parent is set to -1 and each internal node's arrival flag is cleared here,
// so no separate reset pass is needed.
__global__ void k_b_karras(const jt_seg_dev* __restrict__ segs, const int64_t* __restrict__ iprefix,
                           int nseg, const int* __restrict__ segflag)
{
    int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= iprefix[nseg]) return;
    const int g = jt_find(iprefix, nseg, q);
    if (segflag && !segflag[g]) return;   // no particle of this segment needs its tree
    const int64_t i = q - iprefix[g];
    const jt_seg_dev& S = segs[g];
    const jt_tree_dev& T = S.tree;
    const int64_t n = S.n;
    const uint32_t* m30 = T.m30;
    int64_t first, last;
    if (i == 0) {
        first = 0;
        last = n - 1;
        T.parent[0] = -1;
    } else {
        int dl = tdelta(m30, nullptr, n, i, i - 1);
        int dr = tdelta(m30, nullptr, n, i, i + 1);
        int d = (dr > dl) ? 1 : -1;
        int dmin = (d > 0) ? dl : dr;
        int64_t lmax = 2;
        while (tdelta(m30, nullptr, n, i, i + lmax * d) > dmin) lmax *= 2;
        int64_t l = 0;
        for (int64_t t = lmax / 2; t >= 1; t /= 2)
            if (tdelta(m30, nullptr, n, i, i + (l + t) * d) > dmin) l += t;
        int64_t j = i + l * d;
        first = d > 0 ? i : j;
        last = d > 0 ? j : i;
    }
    int64_t gamma = first;
    if (first != last) {
        int dn = tdelta(m30, nullptr, n, first, last);
        int64_t s = 0, t = last - first;
        while (t > 1) {
            t = (t + 1) / 2;
            if (tdelta(m30, nullptr, n, first, first + s + t) > dn) s += t;
        }
        gamma = first + s;
    }
    int64_t lc = (first == gamma) ? (n - 1 + first) : gamma;
    int64_t rc = (gamma + 1 == last) ? (n - 1 + last) : (gamma + 1);
    T.child[i] = make_int2((int)lc, (int)rc);
    T.range[i] = make_int2((int)first, (int)last);
    T.flag[i] = 0;
    T.parent[lc] = (int)i;
    T.parent[rc] = (int)i;
}

// leaves of every segment (particle masses from the box table)
__global__ void k_b_moments(const jt_seg_dev* __restrict__ segs, const jt_box_dev* __restrict__ boxes,
                            const int64_t* __restrict__ pprefix, int nseg, const int* __restrict__ segflag)
{
    int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= pprefix[nseg]) return;
    const int g = jt_find(pprefix, nseg, q);
    if (segflag && !segflag[g]) return;
    const int64_t j = q - pprefix[g];
    const jt_seg_dev& S = segs[g];
    const jt_tree_dev& T = S.tree;
    const int64_t n = S.n;
    const float mass = boxes[S.box].mass[S.species];
    int64_t node = n - 1 + j;
    float4 p = S.pos[j];
    T.com[node] = make_float4(p.x, p.y, p.z, mass);
    T.bmin[node] = make_float4(p.x, p.y, p.z, 0.0f);
    T.bmax[node] = make_float4(p.x, p.y, p.z, 0.0f);
    T.quad0[node] = make_float4(0.f, 0.f, 0.f, 0.f);
    T.quad1[node] = make_float2(0.f, 0.f);
    int cur = n > 1 ? T.parent[node] : -1;
    while (cur >= 0) {
        __threadfence();
        if (atomicAdd(&T.flag[cur], 1) == 0) return;
        int2 ch = __ldcg(&T.child[cur]);
        float4 cl = __ldcg(&T.com[ch.x]);
        float4 cr = __ldcg(&T.com[ch.y]);
        float ml = cl.w, mr = cr.w, m = ml + mr;
        float inv = 1.0f / m;
        float cx = (ml * cl.x + mr * cr.x) * inv;
        float cy = (ml * cl.y + mr * cr.y) * inv;
        float cz = (ml * cl.z + mr * cr.z) * inv;
        float4 lo_l = __ldcg(&T.bmin[ch.x]), lo_r = __ldcg(&T.bmin[ch.y]);
        float4 hi_l = __ldcg(&T.bmax[ch.x]), hi_r = __ldcg(&T.bmax[ch.y]);
        float4 ql0 = __ldcg(&T.quad0[ch.x]), qr0 = __ldcg(&T.quad0[ch.y]);
        float2 ql1 = __ldcg(&T.quad1[ch.x]), qr1 = __ldcg(&T.quad1[ch.y]);
        float dlx = cl.x - cx, dly = cl.y - cy, dlz = cl.z - cz;
        float drx = cr.x - cx, dry = cr.y - cy, drz = cr.z - cz;
        float4 q0;
        q0.x = ql0.x + qr0.x + ml * dlx * dlx + mr * drx * drx;
        q0.y = ql0.y + qr0.y + ml * dly * dly + mr * dry * dry;
        q0.z = ql0.z + qr0.z + ml * dlz * dlz + mr * drz * drz;
        q0.w = ql0.w + qr0.w + ml * dlx * dly + mr * drx * dry;
        float2 q1;
        q1.x = ql1.x + qr1.x + ml * dlx * dlz + mr * drx * drz;
        q1.y = ql1.y + qr1.y + ml * dly * dlz + mr * dry * drz;
        T.com[cur] = make_float4(cx, cy, cz, m);
        T.bmin[cur] = make_float4(fminf(lo_l.x, lo_r.x), fminf(lo_l.y, lo_r.y), fminf(lo_l.z, lo_r.z), 0.0f);
        T.bmax[cur] = make_float4(fmaxf(hi_l.x, hi_r.x), fmaxf(hi_l.y, hi_r.y), fmaxf(hi_l.z, hi_r.z), 0.0f);
        T.quad0[cur] = q0;
        T.quad1[cur] = q1;
        cur = T.parent[cur];
    }
}

}  // namespace

void jt_b_build_trees(const jt_seg_dev* d_segs, const jt_box_dev* d_boxes, int nseg,
                      const int64_t* d_iprefix, int64_t ninternal, const int64_t* d_pprefix,
                      int64_t nleaves, cudaStream_t st, const int* segflag)
{
    if (ninternal > 0)
        k_b_karras<<<(unsigned)((ninternal + 255) / 256), 256, 0, st>>>(d_segs, d_iprefix, nseg, segflag);
    if (nleaves > 0)
        k_b_moments<<<(unsigned)((nleaves + 255) / 256), 256, 0, st>>>(d_segs, d_boxes, d_pprefix, nseg,
                                                                        segflag);
}
