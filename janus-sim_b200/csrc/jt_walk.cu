// Short-range tree walk (+ PM interpolation, + kick), and the step kernels.
//
// ACCURATE walk (k_walk_acc): one warp per group of 32 Morton-consecutive
// target particles of one species; both species' trees are walked in the same
// launch.  The warp tests up to 32 nodes at once (breadth-batched traversal
// from a per-warp stack in shared memory): a node whose AABB lies farther than
// r_cut from the group's AABB (periodic) is dropped; a leaf becomes a direct
// interaction; an internal node whose size l satisfies l < theta * d, with d
// the distance from the group's AABB to the node's centre of mass, becomes a
// monopole + quadrupole interaction; otherwise its two children are pushed.
// Accepted entries are compacted with ballots into shared-memory lists that
// all 32 lanes evaluate against their own particle once 32 entries are
// queued.  Far-field (node) sums are Kahan-compensated.  The PM acceleration
// is interpolated first (CIC of the three force grids) and the kick is
// applied in the epilogue, so acc is written once.
//
// Pair force (G folded into m):  a_i += s_i s_j m_j S(r_p) r / r_p^3 for
// |r| < r_cut, r_p^2 = r^2 + eps^2, S(x) = erfc(x) + 2x/sqrt(pi) e^{-x^2},
// x = r_p/(2 r_s): the exact short-range complement of the Gaussian-filtered
// PM force.  The reference (src/nbody_gpu_twopass.rs:1776-1785) uses erfc(x)
// alone, which drops 0.42 of the Newtonian force at r = 2 r_s.
//
// RCOMPAT walk (k_walk_rc): the reference's forces_treepm_short_range
// (:1670-1811) semantics for 32 particles of the caller-order array per warp:
// one node at a time from a 128-entry stack (pushes only while sp < 127);
// skip when every lane has r - hs > r_cut; monopole when every lane accepts
// (leaf or 4 hs^2 < theta^2 r^2); otherwise descend.  Float expressions are
// evaluated without contraction, in the reference's order.
#include "jt_internal.cuh"

#include <cuda_fp16.h>

#include <cmath>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <vector>
#include <cstdio>

namespace {

constexpr int kWarps = JT_WARPS_PER_BLOCK;
#ifndef JT_WALK_STACK
#define JT_WALK_STACK 384
#endif
constexpr int kStackCap = JT_WALK_STACK;   // per-warp traversal stack (node ids)
constexpr int kRangeCap = 64;     // queued ranges
constexpr int kCandCap = 64;      // candidate particle buffer
constexpr int kApproxCap = 64;    // queued multipole nodes

struct WalkWarpSmem {
    int stack[kStackCap];
    int2 rng[kRangeCap];          // (first sorted index, count)
    char4 rsh[kRangeCap];         // periodic shift of the range, in box lengths (-1, 0, 1)
    float4 cand[kCandCap];        // shifted candidate positions
    // the same candidates relative to the group centre in fp16 (x, y, z
    // arrays; pairs read as half2) for the two-at-a-time distance mask
    __align__(16) __half hc[3][kCandCap];
    float4 acom[kApproxCap];      // shifted COM + mass
    float4 aq0[kApproxCap];       // Qxx Qyy Qzz Qxy
    float2 aq1[kApproxCap];       // Qxz Qyz
};

struct Acc3 {
    float x, y, z;
};

// Phase counters of a diagnostic build (-DJT_WALK_COUNT): traversal
// iterations, ranges streamed, chunks evaluated, pair-loop trip counts (the
// warp's maximum over lanes).  Compiled out of the product build.
struct WalkCount {
    unsigned long long iters, ranges, chunks, trips;
    bool dense;   // the warp's previous full chunk was dense (eval_chunk)
};


__device__ __forceinline__ void kahan_add(float& s, float& c, float v)
{
    float y = v - c;
    float t = s + y;
    c = (t - s) - y;
    s = t;
}

__device__ __forceinline__ float warp_min(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ float warp_max(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

__device__ __forceinline__ float gap1(float d, float ext)
{
    float g = fabsf(d) - ext;
    return g > 0.0f ? g : 0.0f;
}

// Pair forces of both walks read a log-indexed table of the split kernel,
// G(y) = S(sqrt y) / y^{3/2} with y = (r_p / 2 r_s)^2 (JT_LTAB_N entries,
// jt_internal.cuh): the force of a pair is s_i s_j m_j c^3 G(y) d,
// c = 1 / (2 r_s).  One L1-resident float2 load and one FMA replace the
// reciprocal square root, the exp and the reciprocal of the closed form.
// Filled once per device from the host's erfc and exp.
// the cell walk's log-indexed table of G(y) = S(sqrt y) / y^{3/2}
__device__ float2 g_ltab[JT_LTAB_N];

// Fill a log-indexed table of G(y) = S(sqrt y) / y^{3/2} (JT_LTAB_N entries):
// octave e = -32..5, segment k = 0..511 covers [2^e (1 + k/512),
// 2^e (1 + (k+1)/512)); entry (a, b) is the chord through G at its two
// ends, so that G ~ a + b y inside it (relative error <= (h / y)^2 / 8 times
// y^2 |G''| / G: about 2e-6 where G ~ y^{-3/2}, up to ~2e-5 at y ~ 5 where S
// falls off as e^{-y}).  The last entry is the one every y >= 64 (and every
// y < 2^-32, through the unsigned index wrap) is clamped to: S ~ 1e-28 there.
template <class F>
void fill_log_table(F S, float2* tab)
{
    for (int e = -32; e < 6; e++) {
        const double base = std::ldexp(1.0, e), h = base / 512.0;
        for (int k = 0; k < 512; k++) {
            const double y0 = base + k * h, y1 = y0 + h;
            const double g0 = S(y0) / (y0 * std::sqrt(y0)), g1 = S(y1) / (y1 * std::sqrt(y1));
            const double b = (g1 - g0) / h, a = g0 - b * y0;
            tab[(e + 32) * 512 + k] = make_float2((float)a, (float)b);
        }
    }
    tab[JT_LTAB_N - 1] = make_float2(0.f, 0.f);
}

struct WalkArgs {
    const jt_seg_dev* segs;
    const jt_box_dev* boxes;
    const int64_t* gprefix;   // 32-particle groups per segment
    int nseg;
    int parts;                // JT_PART_* bits
    jt_tree_dev pool;         // base of every tree array: a segment's tree is
                              // pool + its node offset (range: + particle offset)
    float kick_frac;          // closing kick fused into the epilogue: this fraction
                              // of each box's dt (0 = none)
    unsigned long long* stats;
    unsigned* err;
    const int64_t* pprefix;       // particles per segment
    const unsigned char* tflag;   // non-null: only flagged particles are computed here
    const int* segflag;           // with tflag: per segment, some particle is flagged
    const float4* pmacc;          // non-null: PM accelerations of the pass (jt_b_interp)
    int64_t npart;                // particles of the pass (pmacc's grid stride)
};

// Pair interactions of this lane's target with a chunk of candidates: a
// distance mask first (8 flops per candidate, fully unrolled for a full chunk
// of 32), then the split-force kernel only for candidates inside r_cut.
// WRAP applies the minimum image per pair (groups wider than L/8; otherwise
// candidates were shifted to the group's image when queued).
template <bool WRAP, int CNT>
__device__ __forceinline__ unsigned chunk_mask(const float4* __restrict__ cand, int cnt, float px,
                                               float py, float pz, const jt_walk_params& P)
{
    unsigned m = 0;
#pragma unroll
    for (int j = 0; j < (CNT > 0 ? CNT : 32); j++) {
        if (CNT == 0 && j >= cnt) break;
        float4 q = cand[j];
        float dx = q.x - px, dy = q.y - py, dz = q.z - pz;
        if (WRAP) {
            dx = jt_wrap(dx, P.L, P.halfL);
            dy = jt_wrap(dy, P.L, P.halfL);
            dz = jt_wrap(dz, P.L, P.halfL);
        }
        float r2 = dx * dx + dy * dy + dz * dz;
        if (r2 < P.rc2) m |= 1u << j;
    }
    return m;
}

// Distance mask of a full chunk from the fp16 copies, two candidates per
// instruction, against a cut inflated to cover fp16 rounding (rch2); the
// evaluation loop re-tests every hit in FP32.  Candidates whose fp16
// coordinate overflows become inf and fail the test, and they are far.
#ifndef JT_WALK_HALF
#define JT_WALK_HALF 1
#endif
// a full chunk whose busiest lane has at least this many hits is evaluated
// densely (eval_chunk)
#ifndef JT_WALK_DENSE
#define JT_WALK_DENSE 22
#endif
__device__ __forceinline__ unsigned chunk_mask_h(const WalkWarpSmem& S, __half2 tx, __half2 ty,
                                                 __half2 tz, __half2 rch2)
{
    const __half2* __restrict__ hx = reinterpret_cast<const __half2*>(S.hc[0]);
    const __half2* __restrict__ hy = reinterpret_cast<const __half2*>(S.hc[1]);
    const __half2* __restrict__ hz = reinterpret_cast<const __half2*>(S.hc[2]);
    unsigned m = 0;
#pragma unroll
    for (int k = 0; k < 16; k++) {
        const __half2 dx = __hsub2(hx[k], tx), dy = __hsub2(hy[k], ty), dz = __hsub2(hz[k], tz);
        const __half2 r2 = __hfma2(dz, dz, __hfma2(dy, dy, __hmul2(dx, dx)));
        const unsigned mk = __hlt2_mask(r2, rch2);          // 0xFFFF per true half
        m |= ((mk & 1u) | ((mk >> 15) & 2u)) << (2 * k);
    }
    return m;
}

struct HalfTarget {
    __half2 tx, ty, tz, rch2;
    bool on;                      // fp16 mask usable for this group
};

// Dense evaluation of a full chunk: every lane takes all 32 candidates, the
// table read predicated by the cut.  Returns the lane's hits.
template <bool WRAP>
__device__ __forceinline__ int eval_dense(const float4* __restrict__ cand, float px, float py, float pz,
                                          bool valid, const jt_walk_params& P, float fac, Acc3& a,
                                          const float2* __restrict__ tab)
{
    int hits = 0;
#pragma unroll 4
    for (int j = 0; j < 32; j++) {
        const float4 q = cand[j];
        const float dx = q.x - px, dy = q.y - py, dz = q.z - pz;
        const float r2 = dx * dx + dy * dy + dz * dz;
        const bool in = valid && r2 > 0.0f && r2 < P.rc2;
        const float y = (r2 + P.eps2) * P.c2;
        const unsigned k = (__float_as_uint(y) >> 14) - JT_LTAB_BASE;   // in range inside the cut
        float2 ab = make_float2(0.f, 0.f);
        if (in) ab = __ldg(&tab[k]);
        const float g = fac * fmaf(ab.y, y, ab.x);
        hits += in ? 1 : 0;
        a.x += g * dx;
        a.y += g * dy;
        a.z += g * dz;
    }
    return hits;
}

__device__ __forceinline__ int warp_max_int(int v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

template <bool WRAP>
__device__ __forceinline__ int eval_chunk(WalkWarpSmem& S, int cnt, int lane, float px, float py,
                                          float pz, bool valid, const jt_walk_params& P, float fac,
                                          WalkCount& wc, Acc3& a, const HalfTarget& H,
                                          const float2* __restrict__ tab)
{
    wc.chunks++;
    (void)lane;
    const float4* __restrict__ cand = S.cand;
    // dense chunks (a clump inside the cut): every lane evaluates all 32
    // candidates instead of looping over its own hits (the warp would run the
    // longest loop anyway, with a branch per hit).  Chunks come in spatial
    // runs, so a chunk after a dense one is evaluated densely at once, without
    // the hit mask, and its own busiest lane decides for the next; the sums
    // are the same either way (out-of-cut candidates add exactly 0)
    if (!WRAP && cnt == 32 && wc.dense) {
        const int hits = eval_dense<WRAP>(cand, px, py, pz, valid, P, fac, a, tab);
        wc.dense = warp_max_int(hits) >= JT_WALK_DENSE;
        return hits;
    }
    unsigned m;
    if (!WRAP && JT_WALK_HALF && cnt == 32 && H.on)
        m = chunk_mask_h(S, H.tx, H.ty, H.tz, H.rch2);
    else
        m = cnt == 32 ? chunk_mask<WRAP, 32>(cand, 32, px, py, pz, P)
                      : chunk_mask<WRAP, 0>(cand, cnt, px, py, pz, P);
    if (!valid) m = 0;
#ifdef JT_WALK_COUNT
    {
        int t = __popc(m);
        for (int o = 16; o > 0; o >>= 1) t = max(t, __shfl_xor_sync(0xffffffffu, t, o));
        wc.trips += t;
    }
#endif
    int hits = 0;
    if (!WRAP && cnt == 32) {
        wc.dense = warp_max_int(__popc(m)) >= JT_WALK_DENSE;
        if (wc.dense) return eval_dense<WRAP>(cand, px, py, pz, valid, P, fac, a, tab);
    }
    while (m) {
        const int j = __ffs(m) - 1;
        m &= m - 1;
        const float4 q = cand[j];
        float dx = q.x - px, dy = q.y - py, dz = q.z - pz;
        if (WRAP) {
            dx = jt_wrap(dx, P.L, P.halfL);
            dy = jt_wrap(dy, P.L, P.halfL);
            dz = jt_wrap(dz, P.L, P.halfL);
        }
        const float r2 = dx * dx + dy * dy + dz * dz;
        if (r2 > 0.0f && r2 < P.rc2) {   // not the target itself; inside the cut
            hits++;
            // fac carries s_i s_j m_j c^3: the force is fac G(y) d
            const float y = (r2 + P.eps2) * P.c2;
            const unsigned k = (__float_as_uint(y) >> 14) - JT_LTAB_BASE;   // in range inside the cut
            const float2 ab = __ldg(&tab[k]);
            const float g = fac * fmaf(ab.y, y, ab.x);
            a.x += g * dx;
            a.y += g * dy;
            a.z += g * dz;
        }
    }
    return hits;
}

// multipole (monopole + quadrupole) interactions, Kahan-compensated
template <bool WRAP>
__device__ __forceinline__ int eval_approx(const float4* __restrict__ cm, const float4* __restrict__ q0s,
                                           const float2* __restrict__ q1s, int cnt, float px, float py,
                                           float pz, bool valid, const jt_walk_params& P, float sgn,
                                           Acc3& s, Acc3& c)
{
    int hits = 0;
    for (int j = 0; j < cnt; j++) {
        float4 m = cm[j];
        float dx = m.x - px, dy = m.y - py, dz = m.z - pz;
        if (WRAP) {
            dx = jt_wrap(dx, P.L, P.halfL);
            dy = jt_wrap(dy, P.L, P.halfL);
            dz = jt_wrap(dz, P.L, P.halfL);
        }
        float r2 = dx * dx + dy * dy + dz * dz;
        if (valid && r2 < P.rc2) {
            hits++;
            float rp2 = r2 + P.eps2;
            float ri = rsqrtf(rp2);
            float x = rp2 * ri * P.c;
            jt_sfac f = jt_split_S2(x, P.c);
            float ri2 = ri * ri, ri3 = ri2 * ri;
            float g = f.S * ri3;
            float G1 = (f.dS - 3.0f * f.S * ri) * ri2 * ri2;
            float G2 = (f.d2S - 7.0f * f.dS * ri + 15.0f * f.S * ri2) * ri2 * ri3;
            float4 a = q0s[j];  // xx yy zz xy
            float2 b = q1s[j];  // xz yz
            float qx = a.x * dx + a.w * dy + b.x * dz;
            float qy = a.w * dx + a.y * dy + b.y * dz;
            float qz = b.x * dx + b.y * dy + a.z * dz;
            float dqd = dx * qx + dy * qy + dz * qz;
            float tr = a.x + a.y + a.z;
            float coef = sgn * (m.w * g + 0.5f * G1 * tr + 0.5f * G2 * dqd);
            float g1s = sgn * G1;
            kahan_add(s.x, c.x, coef * dx + g1s * qx);
            kahan_add(s.y, c.y, coef * dy + g1s * qy);
            kahan_add(s.z, c.z, coef * dz + g1s * qz);
        }
    }
    return hits;
}

// Stream the queued ranges [0, nr) into the candidate buffer, evaluating every
// full chunk of 32.  The next range's particles are loaded while the current
// one is appended (one coalesced float4 load per lane per range).
template <bool WRAP>
__device__ __forceinline__ void drain_ranges(WalkWarpSmem& S, int nr, int& nc,
                                             const float4* __restrict__ tpos, int lane, float px,
                                             float py, float pz, bool valid, const jt_walk_params& P,
                                             float fac, Acc3& near, unsigned& pairs,
                                             unsigned& cands, WalkCount& wc, float gcx, float gcy,
                                             float gcz, float ghx, float ghy, float ghz,
                                             const HalfTarget& H, const float2* __restrict__ tab)
{
    if (nr <= 0) return;
    wc.ranges += nr;
    const unsigned lt = (1u << lane) - 1u;
    int2 r0 = S.rng[0];
    float4 nxt = lane < r0.y ? tpos[r0.x + lane] : make_float4(0.f, 0.f, 0.f, 0.f);
    for (int r = 0; r < nr; r++) {
        const int2 rr = S.rng[r];
        const char4 sc = S.rsh[r];
        const float4 sh = make_float4(sc.x * P.L, sc.y * P.L, sc.z * P.L, 0.f);
        const float4 cur = nxt;
        if (r + 1 < nr) {
            const int2 rn = S.rng[r + 1];
            nxt = lane < rn.y ? tpos[rn.x + lane] : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        // keep only the candidates within r_cut of the group's AABB (no
        // target can reach the others); the box is padded by P.slack and the
        // cut by P.rc2_keep so that float rounding never drops a pair the
        // evaluation would accept
        const float4 c = make_float4(cur.x + sh.x, cur.y + sh.y, cur.z + sh.z, 0.f);
        bool keep = false;
        if (lane < rr.y) {
            float dx = c.x - gcx, dy = c.y - gcy, dz = c.z - gcz;
            if (WRAP) {
                dx = jt_wrap(dx, P.L, P.halfL);
                dy = jt_wrap(dy, P.L, P.halfL);
                dz = jt_wrap(dz, P.L, P.halfL);
            }
            const float gx = gap1(dx, ghx + P.slack), gy = gap1(dy, ghy + P.slack),
                        gz = gap1(dz, ghz + P.slack);
            keep = gx * gx + gy * gy + gz * gz <= P.rc2_keep;
        }
        const unsigned km = __ballot_sync(0xffffffffu, keep);
        if (keep) {
            const int at = nc + __popc(km & lt);
            S.cand[at] = c;
            if (!WRAP && JT_WALK_HALF) {
                S.hc[0][at] = __float2half_rn(c.x - gcx);
                S.hc[1][at] = __float2half_rn(c.y - gcy);
                S.hc[2][at] = __float2half_rn(c.z - gcz);
            }
        }
        nc += __popc(km);
        __syncwarp();
        if (nc >= 32) {
            pairs += eval_chunk<WRAP>(S, 32, lane, px, py, pz, valid, P, fac, wc, near, H, tab);
            cands += 32;
            __syncwarp();
            float4 t = S.cand[32 + lane];
            __half h0 = S.hc[0][32 + lane], h1 = S.hc[1][32 + lane], h2 = S.hc[2][32 + lane];
            __syncwarp();
            if (lane < nc - 32) {
                S.cand[lane] = t;
                S.hc[0][lane] = h0;
                S.hc[1][lane] = h1;
                S.hc[2][lane] = h2;
            }
            nc -= 32;
            __syncwarp();
        }
    }
}

// SCR: the pass holds a screened box; the other species' tree of a screened
// box is walked with the Yukawa table and without multipoles (their
// expansion is of the Newtonian kernel), i.e. every pair inside r_cut
template <int ORDER, int NG, bool WRAP, int BKT, bool SCR>
__device__ __forceinline__ void walk_trees(const WalkArgs& A, const jt_box_dev& B,
                                           const jt_walk_params& P, WalkWarpSmem& S, int s, int lane,
                                           const float4& p, bool valid, float gcx, float gcy,
                                           float gcz, float ghx, float ghy, float ghz, Acc3& near,
                                           Acc3& far, Acc3& comp, unsigned& pairs,
                                           unsigned& nodes, unsigned& cands,
                                           WalkCount& wc)
{
    const unsigned lt = (1u << lane) - 1u;
    // fp16 distance mask: coordinates relative to the group centre; the cut
    // is widened by the rounding of |coordinate| <= D (group half-diagonal
    // + r_cut) on both sides and of the sum of squares
    HalfTarget H;
    {
        const float D = sqrtf(ghx * ghx + ghy * ghy + ghz * ghz) + P.rc;
        const float rl = (P.rc + 8.0f * 4.8828125e-4f * (D + P.rc)) * (1.0f + 8.0f * 4.8828125e-4f);
        H.on = rl * rl < 3.0e4f;
        H.tx = __float2half2_rn(p.x - gcx);
        H.ty = __float2half2_rn(p.y - gcy);
        H.tz = __float2half2_rn(p.z - gcz);
        H.rch2 = __float2half2_rn(rl * rl);
    }
    for (int t = 0; t < 2; t++) {
        const int tg = B.seg[t];
        if (tg < 0 || !(P.parts & 2)) continue;
        const jt_seg_dev& TS = A.segs[tg];
        const int nt = (int)TS.n;   // < 2^30 per species
        if (nt == 0) continue;
        // node arrays through the pool bases (kernel parameters, no
        // registers) plus two 32-bit offsets
        const int noff = (int)(TS.tree.com - A.pool.com);
        const int roff = (int)(TS.tree.range - A.pool.range);
        const float4* __restrict__ tpos = TS.pos;
        const float sgn = (s == t) ? 1.0f : -1.0f;
        // no dynamic index into a local array (P.mass carries the table's c^3)
        const float fac_direct = sgn * (t == 0 ? P.mass[0] : P.mass[1]);
        const bool yuk = SCR && s != t && B.ytab != nullptr;
        const float2* __restrict__ tab = yuk ? B.ytab : g_ltab;
        const float theta2 = yuk ? 0.0f : P.theta2;
        const int leaf0 = nt - 1;
        int sp = 1, nR = 0, nA = 0, nc = 0;
        if (lane == 0) S.stack[0] = 0;
        __syncwarp();
        while (sp > 0) {
            wc.iters++;
            const int k = sp < 32 ? sp : 32;
            int node = lane < k ? S.stack[sp - k + lane] : -1;
            sp -= k;
            __syncwarp();
            if (node >= 2 * nt - 1) {  // never expected: keeps a corrupted id off the loads
                atomicOr(A.err, JT_ERRBIT_STACK);
                node = -1;
            }
            int act = 0;  // 1 open, 2 range, 3 multipole
            float4 pay = make_float4(0.f, 0.f, 0.f, 0.f), pq0 = pay;
            float2 pq1 = make_float2(0.f, 0.f);
            int2 ch = make_int2(0, 0), rg = make_int2(0, 0);
            if (node >= 0) {
                float lox, loy, loz, hix, hiy, hiz;
                int first, count;
                float4 cmv = make_float4(0.f, 0.f, 0.f, 0.f);
                int2 chv = make_int2(0, 0);
                if (node >= leaf0) {
                    first = (int)(node - leaf0);
                    count = 1;
                    float4 q = tpos[first];
                    lox = hix = q.x; loy = hiy = q.y; loz = hiz = q.z;
                } else {
                    // every array of an internal node is loaded at once: one
                    // memory latency per traversal step instead of three
                    int2 r = A.pool.range[roff + node];
                    float4 lo = A.pool.bmin[noff + node], hi = A.pool.bmax[noff + node];
                    cmv = A.pool.com[noff + node];
                    chv = A.pool.child[noff + node];
                    first = r.x;
                    count = r.y - r.x + 1;
                    lox = lo.x; loy = lo.y; loz = lo.z; hix = hi.x; hiy = hi.y; hiz = hi.z;
                }
                float nhx = 0.5f * (hix - lox), nhy = 0.5f * (hiy - loy), nhz = 0.5f * (hiz - loz);
                float cx = 0.5f * (hix + lox), cy = 0.5f * (hiy + loy), cz = 0.5f * (hiz + loz);
                float dx = jt_wrap(cx - gcx, P.L, P.halfL);
                float dy = jt_wrap(cy - gcy, P.L, P.halfL);
                float dz = jt_wrap(cz - gcz, P.L, P.halfL);
                float gx = gap1(dx, ghx + nhx), gy = gap1(dy, ghy + nhy), gz = gap1(dz, ghz + nhz);
                if (gx * gx + gy * gy + gz * gz <= P.rc2) {
                    bool accepted = false;
                    if (count > 1) {
                        const float4 cm = cmv;
                        float mx = jt_wrap(cm.x - gcx, P.L, P.halfL);
                        float my = jt_wrap(cm.y - gcy, P.L, P.halfL);
                        float mz = jt_wrap(cm.z - gcz, P.L, P.halfL);
                        float ax = gap1(mx, ghx), ay = gap1(my, ghy), az = gap1(mz, ghz);
                        float dm2 = ax * ax + ay * ay + az * az;
                        float size = 2.0f * fmaxf(fmaxf(nhx, nhy), nhz);
                        if (size * size < theta2 * dm2) {
                            accepted = true;
                            act = 3;
                            pay = make_float4(gcx + mx, gcy + my, gcz + mz, cm.w);
                            pq0 = A.pool.quad0[noff + node];
                            pq1 = A.pool.quad1[noff + node];
                        }
                    }
                    if (!accepted) {
                        if (count <= BKT) {
                            act = 2;
                            rg = make_int2(first, count);
                            // shift (in box lengths) that moves the node to the group's image
                            pay = make_float4(rintf(((gcx + dx) - cx) / P.L), rintf(((gcy + dy) - cy) / P.L),
                                              rintf(((gcz + dz) - cz) / P.L), 0.f);
                        } else {
                            act = 1;
                            ch = chv;
                        }
                    }
                }
            }
            const unsigned mopen = __ballot_sync(0xffffffffu, act == 1);
            const unsigned mrng = __ballot_sync(0xffffffffu, act == 2);
            const unsigned mapp = __ballot_sync(0xffffffffu, act == 3);
            if (act == 1) {
                int at = sp + 2 * __popc(mopen & lt);
                if (at + 1 < kStackCap) {
                    S.stack[at] = ch.y;
                    S.stack[at + 1] = ch.x;
                } else {
                    atomicOr(A.err, JT_ERRBIT_STACK);
                }
            } else if (act == 2) {
                int at = nR + __popc(mrng & lt);
                S.rng[at] = rg;
                S.rsh[at] = make_char4((signed char)pay.x, (signed char)pay.y, (signed char)pay.z, 0);
            } else if (act == 3) {
                int at = nA + __popc(mapp & lt);
                S.acom[at] = pay;
                S.aq0[at] = pq0;
                S.aq1[at] = pq1;
            }
            {
                int room = (kStackCap - sp) / 2;
                int no = __popc(mopen);
                sp += 2 * (no < room ? no : room);
            }
            nR += __popc(mrng);
            nA += __popc(mapp);
            __syncwarp();
            if (nR >= 32) {
                drain_ranges<WRAP>(S, 32, nc, tpos, lane, p.x, p.y, p.z, valid, P, fac_direct, near,
                                   pairs, cands, wc, gcx, gcy, gcz, ghx, ghy, ghz, H, tab);
                __syncwarp();
                int2 r2 = S.rng[32 + lane];
                char4 s2 = S.rsh[32 + lane];
                __syncwarp();
                if (lane < nR - 32) { S.rng[lane] = r2; S.rsh[lane] = s2; }
                nR -= 32;
                __syncwarp();
            }
            if (nA >= 32) {
                nodes += eval_approx<WRAP>(S.acom, S.aq0, S.aq1, 32, p.x, p.y, p.z, valid, P, sgn, far, comp);
                __syncwarp();
                float4 t0 = S.acom[32 + lane], t1 = S.aq0[32 + lane];
                float2 t2 = S.aq1[32 + lane];
                __syncwarp();
                if (lane < nA - 32) {
                    S.acom[lane] = t0;
                    S.aq0[lane] = t1;
                    S.aq1[lane] = t2;
                }
                nA -= 32;
                __syncwarp();
            }
        }
        drain_ranges<WRAP>(S, nR, nc, tpos, lane, p.x, p.y, p.z, valid, P, fac_direct, near, pairs,
                           cands, wc, gcx, gcy, gcz, ghx, ghy, ghz, H, tab);
        __syncwarp();
        if (nc > 0) {
            pairs += eval_chunk<WRAP>(S, nc, lane, p.x, p.y, p.z, valid, P, fac_direct, wc, near, H, tab);
            cands += nc;
        }
        if (nA > 0)
            nodes += eval_approx<WRAP>(S.acom, S.aq0, S.aq1, nA, p.x, p.y, p.z, valid, P, sgn, far, comp);
        __syncwarp();
    }
}

// PM acceleration of a unit m+ particle at p from one set of force grids
// (SG false, B.force: the signed source's, which an m- particle takes with
// minus sign; SG true, B.force_s: the unsigned source's of a screened box,
// taken by both): the deposit's stencil on every grid (the interlaced grid's
// nodes sit half a cell higher), averaged over the grids
template <int ORDER, int NG, bool SG = false>
__device__ __forceinline__ Acc3 pm_interp(const jt_box_dev& B, const float4& p)
{
    Acc3 pm = {0.f, 0.f, 0.f};
    {
        const int M = B.M, mask = M - 1;
        const int64_t G = (int64_t)M * M * M;
        const float gx = (p.x + B.halfL) * B.h_inv, gy = (p.y + B.halfL) * B.h_inv,
                    gz = (p.z + B.halfL) * B.h_inv;
#pragma unroll
        for (int b = 0; b < NG; b++) {
            const float sh = 0.5f * b;
            float wx[ORDER], wy[ORDER], wz[ORDER];
            const int ix = jt_stencil<ORDER>(gx - sh, wx);
            const int iy = jt_stencil<ORDER>(gy - sh, wy);
            const int iz = jt_stencil<ORDER>(gz - sh, wz);
            const float* __restrict__ F = (SG ? B.force_s : B.force) + (int64_t)b * 3 * G;
#pragma unroll
            for (int c = 0; c < ORDER; c++)
#pragma unroll
                for (int bb = 0; bb < ORDER; bb++) {
                    const float wyz = wz[c] * wy[bb];
                    const int64_t row = ((int64_t)((iz + c) & mask) * M + ((iy + bb) & mask)) * M;
#pragma unroll
                    for (int a = 0; a < ORDER; a++) {
                        const int64_t id = row + ((ix + a) & mask);
                        const float w = wyz * wx[a];
                        pm.x += w * __ldg(F + id);
                        pm.y += w * __ldg(F + G + id);
                        pm.z += w * __ldg(F + 2 * G + id);
                    }
                }
        }
        if (NG == 2) { pm.x *= 0.5f; pm.y *= 0.5f; pm.z *= 0.5f; }
    }

    return pm;
}

// The PM acceleration of a unit m+ particle computed by the tiled
// interpolation kernel (jt_b_interp) for pass particle gi: the mean of the
// interlaced grids' values.
template <int NG>
__device__ __forceinline__ Acc3 pm_from_tiles(const float4* __restrict__ pmacc, int64_t npart, int64_t gi)
{
    float4 a = pmacc[gi];
    if (NG == 2) {
        const float4 b = pmacc[npart + gi];
        a.x = 0.5f * (a.x + b.x);
        a.y = 0.5f * (a.y + b.y);
        a.z = 0.5f * (a.z + b.z);
    }
    return Acc3{a.x, a.y, a.z};
}

// MINB: resident blocks per SM the register budget is sized for (6 -> 80
// registers); BKT: nodes with <= BKT particles are streamed as ranges
// (<= 32: one lane per particle when a range is loaded)
template <int ORDER, int NG, int MINB, int BKT, bool SCR>
__global__ void __launch_bounds__(kWarps * 32, MINB) k_walk_acc(WalkArgs A)
{
    static_assert(BKT <= 32, "a range is loaded one particle per lane");
    __shared__ WalkWarpSmem smem_all[kWarps];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    WalkWarpSmem& S = smem_all[wib];
    const int64_t gw = (int64_t)blockIdx.x * kWarps + wib;
    if (gw >= A.gprefix[A.nseg]) return;  // whole warp
    const int g = jt_find(A.gprefix, A.nseg, gw);
    if (A.segflag && A.segflag[g] == 0) return;   // whole warp: no flagged particle in this segment
    const int64_t grp = gw - A.gprefix[g];
    const jt_seg_dev& SG = A.segs[g];
    const jt_box_dev& B = A.boxes[SG.box];
    const int s = SG.species;
    jt_walk_params P;
    P.L = B.L; P.halfL = B.halfL; P.theta2 = B.theta2; P.c = B.c;
    P.c2 = B.c * B.c;
    // the pair table covers y = (r^2 + eps^2) c^2 in [2^-32, 2^6): a
    // softening below 2^-16 (2 r_s) is raised to it, and the cut is bounded
    // by y < 64 (16 r_s without softening; the split factor is below 1e-27
    // there), so that no pair's table index needs a clamp
    P.eps2 = fmaxf(B.eps2, 2.3285392e-10f / P.c2);
    P.rc2 = fminf(B.rc2, 64.0f * 0.99999f / P.c2 - P.eps2);
    P.rc = sqrtf(P.rc2);
    // particle masses times c^3, the scale of the pair table's G(y)
    P.mass[0] = B.mass[0] * P.c2 * B.c; P.mass[1] = B.mass[1] * P.c2 * B.c;
    // candidate prefilter margins: 8 ulp of the largest coordinate on the
    // box, 1e-5 relative on the cut
    P.slack = B.halfL * 9.5367431640625e-7f;
    P.rc2_keep = B.rc2 * 1.00001f;
    P.M = B.M; P.h_inv = B.h_inv; P.order = ORDER; P.ngrid = NG; P.parts = A.parts;
    const int64_t ns = SG.n;
    const int64_t i = grp * 32 + lane;
    const bool valid = i < ns;
    // with a cell walk before this one, only its flagged particles are left
    const bool mine = !A.tflag || (valid && A.tflag[A.pprefix[g] + i]);
    if (A.tflag && !__any_sync(0xffffffffu, mine)) return;
    const float4 p = SG.pos[valid ? i : grp * 32];
    const float sgn_s = s == 0 ? 1.0f : -1.0f;

    // group AABB
    float lox = warp_min(p.x), loy = warp_min(p.y), loz = warp_min(p.z);
    float hix = warp_max(p.x), hiy = warp_max(p.y), hiz = warp_max(p.z);
    float gcx = 0.5f * (lox + hix), gcy = 0.5f * (loy + hiy), gcz = 0.5f * (loz + hiz);
    float ghx = 0.5f * (hix - lox), ghy = 0.5f * (hiy - loy), ghz = 0.5f * (hiz - loz);

    Acc3 pm = {0.f, 0.f, 0.f};
    if ((P.parts & 1) && !A.pmacc) pm = pm_interp<ORDER, NG>(B, p);

    Acc3 near = {0.f, 0.f, 0.f}, far = {0.f, 0.f, 0.f}, comp = {0.f, 0.f, 0.f};
    unsigned pairs = 0, nodes = 0, cands = 0;   // per lane (warp totals < 2^32)
    WalkCount wc = {0, 0, 0, 0, false};
    // groups wider than L/8 take the minimum image per pair
    const bool wide = fmaxf(fmaxf(ghx, ghy), ghz) > 0.125f * P.L;
    if (wide)
        walk_trees<ORDER, NG, true, BKT, SCR>(A, B, P, S, s, lane, p, valid, gcx, gcy, gcz, ghx, ghy, ghz, near,
                                    far, comp, pairs, nodes, cands, wc);
    else
        walk_trees<ORDER, NG, false, BKT, SCR>(A, B, P, S, s, lane, p, valid, gcx, gcy, gcz, ghx, ghy, ghz, near,
                                     far, comp, pairs, nodes, cands, wc);

    if (valid && mine) {
        if ((P.parts & 1) && A.pmacc) pm = pm_from_tiles<NG>(A.pmacc, A.npart, A.pprefix[g] + i);
        float ax = sgn_s * pm.x + near.x + (far.x - comp.x);
        float ay = sgn_s * pm.y + near.y + (far.y - comp.y);
        float az = sgn_s * pm.z + near.z + (far.z - comp.z);
        if (SCR && B.force_s && (P.parts & 1)) {
            const Acc3 ps = pm_interp<ORDER, NG, true>(B, p);
            ax += ps.x;
            ay += ps.y;
            az += ps.z;
        }
        SG.acc[i] = make_float4(ax, ay, az, 0.f);
        if (A.kick_frac != 0.0f) {
            // kick_frac 0.5: the closing half kick; 1.0: the closing half
            // kick and the next step's opening half kick, applied one after
            // the other (with drag, one full kick would differ by O(H a dt^2)
            // and make a trajectory depend on how steps are grouped in calls)
            const float drag = B.kick_drag, h = 0.5f * B.dt;
            float4 v = SG.vel[i];
            v.x += (ax - drag * v.x) * h;
            v.y += (ay - drag * v.y) * h;
            v.z += (az - drag * v.z) * h;
            if (A.kick_frac > 0.75f) {
                v.x += (ax - drag * v.x) * h;
                v.y += (ay - drag * v.y) * h;
                v.z += (az - drag * v.z) * h;
            }
            SG.vel[i] = v;
        }
    }
    if (A.stats) {
        if (!mine) pairs = nodes = 0;   // those lanes' accelerations came from the cell walk
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
            nodes += __shfl_xor_sync(0xffffffffu, nodes, o);
        }
        if (lane == 0) {
            atomicAdd(A.stats, (unsigned long long)pairs);
            atomicAdd(A.stats + 1, (unsigned long long)nodes);
            atomicAdd(A.stats + 2, (unsigned long long)cands * 32ull);
#ifdef JT_WALK_COUNT
            atomicAdd(A.stats + 3, wc.iters);
            atomicAdd(A.stats + 4, wc.ranges);
            atomicAdd(A.stats + 5, wc.chunks);
            atomicAdd(A.stats + 6, wc.trips);
#endif
        }
    }
}

// ------------------------------------------------------------------ RCOMPAT
struct RcArgs {
    jt_rc_params p;
    const float4* pos;      // caller order, both species
    const int8_t* sg;
    int64_t n_all;
    int64_t n[2];
    jt_tree_dev tree[2];
    const float* phi;
    float4* acc;
    unsigned* err;
};

__device__ __forceinline__ float rc_wrap(float d, float bh)
{
    if (d > bh) d = __fsub_rn(d, __fmul_rn(2.0f, bh));
    if (d < -bh) d = __fadd_rn(d, __fmul_rn(2.0f, bh));
    return d;
}

__global__ void __launch_bounds__(kWarps * 32) k_walk_rc(RcArgs A)
{
    __shared__ int stack_all[kWarps][128];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    int* stack = stack_all[wib];
    const int64_t tid = ((int64_t)blockIdx.x * kWarps + wib) * 32 + lane;
    const int64_t wbase = tid - lane;
    if (wbase >= A.n_all) return;  // whole warp
    const jt_rc_params& P = A.p;
    const bool valid = tid < A.n_all;
    const int64_t st = valid ? tid : 0;
    const float4 p = A.pos[st];
    const int my_sign = A.sg[st] > 0 ? 1 : -1;
    float res[2][3] = {{0.f, 0.f, 0.f}, {0.f, 0.f, 0.f}};

    for (int t = 0; t < 2; t++) {
        const int64_t nt = A.n[t];
        if (nt == 0 || !(P.parts & 2)) continue;
        const jt_tree_dev T = A.tree[t];
        const int tree_sign = t == 0 ? 1 : -1;
        const float sf = (my_sign == tree_sign) ? 1.0f : -1.0f;
        float ax = 0.f, ay = 0.f, az = 0.f;
        int sp = 0;
        if (lane == 0) stack[0] = 0;
        sp = 1;
        __syncwarp();
        while (sp > 0) {
            const int node = stack[sp - 1];
            --sp;
            __syncwarp();
            const bool leaf = node >= nt - 1;
            const float4 b = T.bmin[node];   // cx cy cz hs
            const float4 cm = T.com[node];   // comx comy comz m
            float dx = rc_wrap(__fsub_rn(b.x, p.x), P.box_half_q);
            float dy = rc_wrap(__fsub_rn(b.y, p.y), P.box_half_q);
            float dz = rc_wrap(__fsub_rn(b.z, p.z), P.box_half_q);
            float r2 = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(dx, dx), __fmul_rn(dy, dy)),
                                           __fmul_rn(dz, dz)), 1e-20f);
            // the screened walk (:911-1035) has no r_cut prune
            if (!P.screen) {
                float r = __fsqrt_rn(r2);
                bool beyond = __fsub_rn(r, b.w) > P.r_cut;
                if (__all_sync(0xffffffffu, beyond)) continue;
            }
            bool approx = leaf || (__fmul_rn(__fmul_rn(4.0f, b.w), b.w) < __fmul_rn(P.theta2, r2));
            if (__all_sync(0xffffffffu, approx)) {
                if (valid) {
                    float ddx = rc_wrap(__fsub_rn(cm.x, p.x), P.box_half_q);
                    float ddy = rc_wrap(__fsub_rn(cm.y, p.y), P.box_half_q);
                    float ddz = rc_wrap(__fsub_rn(cm.z, p.z), P.box_half_q);
                    float rp2 = __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(ddx, ddx), __fmul_rn(ddy, ddy)),
                                                    __fmul_rn(ddz, ddz)), P.eps2);
                    float rp = __fsqrt_rn(rp2);
                    if (P.screen) {
                        // s_i s_t S m / r_p^3, S = exp(-x)(1 + x), x = r_p / lambda,
                        // for opposite signs (:1000-1017)
                        float irp3 = __fdiv_rn(1.0f, __fmul_rn(rp2, rp));
                        float scr = 1.0f;
                        if (sf < 0.0f && P.inv_lambda > 0.0f) {
                            float x = __fmul_rn(rp, P.inv_lambda);
                            scr = __fmul_rn(expf(-x), __fadd_rn(1.0f, x));
                        }
                        float f = __fmul_rn(__fmul_rn(__fmul_rn(sf, scr), cm.w), irp3);
                        ax = __fadd_rn(ax, __fmul_rn(f, ddx));
                        ay = __fadd_rn(ay, __fmul_rn(f, ddy));
                        az = __fadd_rn(az, __fmul_rn(f, ddz));
                    } else {
                        float arg = __fdiv_rn(rp, __fmul_rn(2.0f, P.r_s));
                        float ef = erfcf(arg);
                        if (ef > 1e-6f) {
                            float irp3 = __fdiv_rn(1.0f, __fmul_rn(rp, rp2));
                            float f = __fmul_rn(__fmul_rn(__fmul_rn(sf, cm.w), irp3), ef);
                            ax = __fadd_rn(ax, __fmul_rn(f, ddx));
                            ay = __fadd_rn(ay, __fmul_rn(f, ddy));
                            az = __fadd_rn(az, __fmul_rn(f, ddz));
                        }
                    }
                }
            } else {
                // not every lane accepts (a leaf is always accepted): lane 0
                // pushes right then left while sp < 127; sp is warp-uniform
                int2 ch = T.child[node];
                if (ch.y >= 0 && sp < 127) { if (lane == 0) stack[sp] = ch.y; ++sp; }
                if (ch.x >= 0 && sp < 127) { if (lane == 0) stack[sp] = ch.x; ++sp; }
            }
            __syncwarp();
        }
        res[t][0] = ax; res[t][1] = ay; res[t][2] = az;
    }

    if (!valid) return;
    // PM: central differences of the signed potential at the 8 CIC nodes
    // (cic_gather, :162-257); F = -s grad(phi)
    const int M = P.M;
    float gx = __fmul_rn(__fadd_rn(p.x, P.box_half), P.inv_cell);
    float gy = __fmul_rn(__fadd_rn(p.y, P.box_half), P.inv_cell);
    float gz = __fmul_rn(__fadd_rn(p.z, P.box_half), P.inv_cell);
    float Mf = (float)M;
    gx = fmodf(__fadd_rn(gx, Mf), Mf);
    gy = fmodf(__fadd_rn(gy, Mf), Mf);
    gz = fmodf(__fadd_rn(gz, Mf), Mf);
    int ix = (int)gx, iy = (int)gy, iz = (int)gz;
    float fx = __fsub_rn(gx, (float)ix), fy = __fsub_rn(gy, (float)iy), fz = __fsub_rn(gz, (float)iz);
    float wx[2] = {__fsub_rn(1.0f, fx), fx}, wy[2] = {__fsub_rn(1.0f, fy), fy},
          wz[2] = {__fsub_rn(1.0f, fz), fz};
    // positions outside the box (or NaN) still index inside the grid
    ix = ((ix % M) + M) % M; iy = ((iy % M) + M) % M; iz = ((iz % M) + M) % M;
    float inv_2h = __fdiv_rn(0.5f, P.cell);
    float sgn = (float)my_sign;
    float Fx = 0.f, Fy = 0.f, Fz = 0.f;
    const float* phi = A.phi;
    if (P.parts & 1)
#define RCIDX(a, b, c) ((int64_t)(a) + (int64_t)M * ((int64_t)(b) + (int64_t)M * (int64_t)(c)))
    for (int di = 0; di < 2; di++)
        for (int dj = 0; dj < 2; dj++)
            for (int dk = 0; dk < 2; dk++) {
                int ci = (ix + di) % M, cj = (iy + dj) % M, ck = (iz + dk) % M;
                float w = __fmul_rn(__fmul_rn(wx[di], wy[dj]), wz[dk]);
                int cip = (ci + 1) % M, cim = (ci + M - 1) % M;
                int cjp = (cj + 1) % M, cjm = (cj + M - 1) % M;
                int ckp = (ck + 1) % M, ckm = (ck + M - 1) % M;
                float ddx = __fmul_rn(__fsub_rn(phi[RCIDX(cip, cj, ck)], phi[RCIDX(cim, cj, ck)]), inv_2h);
                float ddy = __fmul_rn(__fsub_rn(phi[RCIDX(ci, cjp, ck)], phi[RCIDX(ci, cjm, ck)]), inv_2h);
                float ddz = __fmul_rn(__fsub_rn(phi[RCIDX(ci, cj, ckp)], phi[RCIDX(ci, cj, ckm)]), inv_2h);
                Fx = __fadd_rn(Fx, __fmul_rn(w, -__fmul_rn(sgn, ddx)));
                Fy = __fadd_rn(Fy, __fmul_rn(w, -__fmul_rn(sgn, ddy)));
                Fz = __fadd_rn(Fz, __fmul_rn(w, -__fmul_rn(sgn, ddz)));
            }
#undef RCIDX
    // acc = (tree+ + tree-) + pm, the reference's accumulation order
    float ax = __fadd_rn(__fadd_rn(res[0][0], res[1][0]), Fx);
    float ay = __fadd_rn(__fadd_rn(res[0][1], res[1][1]), Fy);
    float az = __fadd_rn(__fadd_rn(res[0][2], res[1][2]), Fz);
    A.acc[tid] = make_float4(ax, ay, az, 0.f);
}

// ------------------------------------------------------------------ step kernels
__global__ void k_kick(float4* __restrict__ vel, const float4* __restrict__ acc, int64_t n, float dt,
                       float drag)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 v = vel[i], a = acc[i];
    v.x += (a.x - drag * v.x) * dt;
    v.y += (a.y - drag * v.y) * dt;
    v.z += (a.z - drag * v.z) * dt;
    vel[i] = v;
}

// drift with one periodic wrap (drift_f32, :33-48)
__global__ void k_drift(float4* __restrict__ pos, const float4* __restrict__ vel, int64_t n, float dt,
                        float L, float halfL)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 p = pos[i], v = vel[i];
    p.x += v.x * dt;
    p.y += v.y * dt;
    p.z += v.z * dt;
    p.x = p.x > halfL ? p.x - L : p.x;
    p.x = p.x < -halfL ? p.x + L : p.x;
    p.y = p.y > halfL ? p.y - L : p.y;
    p.y = p.y < -halfL ? p.y + L : p.y;
    p.z = p.z > halfL ? p.z - L : p.z;
    p.z = p.z < -halfL ? p.z + L : p.z;
    pos[i] = p;
}

__global__ void k_to_caller(const float4* __restrict__ src, const int* __restrict__ id,
                            const int* __restrict__ gmap, int64_t n, float4* __restrict__ dst)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    dst[gmap[id[i]]] = src[i];
}

__global__ void k_aos_out(const float4* __restrict__ src, const int* __restrict__ id,
                          const int* __restrict__ gmap, int64_t n, float* __restrict__ dst)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 v = src[i];
    int64_t k = id ? id[i] : i;
    if (gmap) k = gmap[k];
    int64_t o = 3 * k;
    dst[o] = v.x;
    dst[o + 1] = v.y;
    dst[o + 2] = v.z;
}

__global__ void k_from_caller(const float4* __restrict__ src, const int* __restrict__ id,
                              const int* __restrict__ gmap, int64_t n, float4* __restrict__ dst)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    dst[i] = src[gmap[id[i]]];
}

__global__ void k_aos_in(const float* __restrict__ src, int64_t n, float4* __restrict__ dst,
                         int* __restrict__ id)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    dst[i] = src ? make_float4(src[3 * i], src[3 * i + 1], src[3 * i + 2], 0.f)
                 : make_float4(0.f, 0.f, 0.f, 0.f);
    if (id) id[i] = (int)i;
}

// 256 particles (768 words) per block; the host side is touched only as
// contiguous words t, t + 256, t + 512 of the block's span.
__global__ void __launch_bounds__(256) k_host_in(const float* __restrict__ src, int64_t n,
                                                 float4* __restrict__ dst, int* __restrict__ id)
{
    __shared__ float w[768];
    const int64_t base = (int64_t)blockIdx.x * 256;
    const int m = n - base < 256 ? (int)(n - base) : 256;
    const float* s = src + 3 * base;
    for (int k = threadIdx.x; k < 3 * m; k += 256) w[k] = s[k];
    __syncthreads();
    const int t = threadIdx.x;
    if (t < m) {
        dst[base + t] = make_float4(w[3 * t], w[3 * t + 1], w[3 * t + 2], 0.f);
        if (id) id[base + t] = (int)(base + t);
    }
}

__global__ void k_inverse(const int* __restrict__ id, int64_t n, int* __restrict__ inv)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) inv[id[i]] = (int)i;
}

__global__ void __launch_bounds__(256) k_host_out(const float4* __restrict__ src, const int* __restrict__ inv,
                                                  int64_t n, float* __restrict__ dst)
{
    __shared__ float w[768];
    const int64_t base = (int64_t)blockIdx.x * 256;
    const int m = n - base < 256 ? (int)(n - base) : 256;
    const int t = threadIdx.x;
    if (t < m) {
        float4 v = src[inv[base + t]];
        w[3 * t] = v.x;
        w[3 * t + 1] = v.y;
        w[3 * t + 2] = v.z;
    }
    __syncthreads();
    float* d = dst + 3 * base;
    for (int k = t; k < 3 * m; k += 256) d[k] = w[k];
}

__global__ void k_split_signed(const float* __restrict__ pos, const float* __restrict__ vel,
                               const int8_t* __restrict__ sg, int64_t n, const int* __restrict__ rank,
                               float4* pos_p, float4* vel_p, int* id_p, int* gmap_p, float4* pos_m,
                               float4* vel_m, int* id_m, int* gmap_m)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int r = rank[i];
    float4 p = make_float4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], 0.f);
    float4 v = vel ? make_float4(vel[3 * i], vel[3 * i + 1], vel[3 * i + 2], 0.f)
                   : make_float4(0.f, 0.f, 0.f, 0.f);
    if (sg[i] > 0) {
        pos_p[r] = p; vel_p[r] = v; id_p[r] = r; gmap_p[r] = (int)i;
    } else {
        pos_m[r] = p; vel_m[r] = v; id_m[r] = r; gmap_m[r] = (int)i;
    }
}

}  // namespace

namespace {

// Fill g_ltab on the current device once (host double erfc/exp).
int stab_ready()
{
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return JT_ECUDA;
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev]) return JT_OK;
    auto S = [](double y) {
        const double x = std::sqrt(y);
        return std::erfc(x) + 1.1283791670955126 * x * std::exp(-y);
    };
    std::vector<float2> lt(JT_LTAB_N);
    fill_log_table(S, lt.data());
    if (cudaMemcpyToSymbol(g_ltab, lt.data(), sizeof(float2) * JT_LTAB_N) != cudaSuccess) return JT_ECUDA;
    done[dev] = true;
    return JT_OK;
}

}  // namespace

namespace {

// ---- walk autotuner --------------------------------------------------------
// The default launch shape of the walk (80 registers, 6 blocks per SM,
// 32-particle leaf buckets) is the best measured at 2x224^3; other densities,
// clustering and box mixes can prefer another register budget or bucket.  For
// the default PM scheme (PCS, interlaced) the first force-only pass of each
// size class (device, log2 of the warp-group count) times every variant once
// and keeps the fastest; JT_WALK_VARIANT=<k> pins variant k.  Passes that kick
// (the walk then updates velocities) or run under stream capture use the
// cached or the default variant.
struct WalkVariant {
    int minb, bkt;
};
constexpr WalkVariant kVariants[] = {{6, 32}, {5, 32}, {6, 24}};
constexpr int kNumVariants = sizeof(kVariants) / sizeof(kVariants[0]);

std::mutex g_tune_mu;
std::map<std::pair<int, int>, int> g_tuned;   // (device, log2 groups) -> variant

// the variants of the default PM scheme (PCS, interlaced)
void launch_variant(int v, unsigned g, const WalkArgs& A, cudaStream_t st)
{
    switch (v) {
    case 1: k_walk_acc<4, 2, 5, 32, false><<<g, kWarps * 32, 0, st>>>(A); break;
    case 2: k_walk_acc<4, 2, 6, 24, false><<<g, kWarps * 32, 0, st>>>(A); break;
    default: k_walk_acc<4, 2, 6, 32, false><<<g, kWarps * 32, 0, st>>>(A); break;
    }
}

int pick_variant(unsigned g, int64_t ngroups, const WalkArgs& A, cudaStream_t st)
{
    if (const char* e = std::getenv("JT_WALK_VARIANT")) {
        const int v = std::atoi(e);
        return v >= 0 && v < kNumVariants ? v : 0;
    }
    int dev = 0;
    cudaGetDevice(&dev);
    int lg = 0;
    while (((int64_t)1 << (lg + 1)) <= ngroups) lg++;
    const std::pair<int, int> key(dev, lg);
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) return it->second;
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (A.kick_frac != 0.0f || cudaStreamIsCapturing(st, &cs) != cudaSuccess ||
        cs != cudaStreamCaptureStatusNone)
        return 0;
    // time each variant on this pass (force only: every run writes the same
    // accelerations); statistics are left to the real launch
    WalkArgs T = A;
    T.stats = nullptr;
    cudaEvent_t e0, e1;
    if (cudaEventCreate(&e0) != cudaSuccess) return 0;
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return 0;
    }
    int best = 0;
    float best_ms = 0.f;
    for (int v = 0; v < kNumVariants; v++) {
        cudaEventRecord(e0, st);
        launch_variant(v, g, T, st);
        cudaEventRecord(e1, st);
        float ms = 0.f;
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
            best = 0;
            break;
        }
        if (v == 0 || ms < best_ms) {
            best = v;
            best_ms = ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tuned[key] = best;
    return best;
}

}  // namespace

extern "C" int jt_walk_tuning(char* buf, size_t len)
{
    if (!buf || len == 0) return JT_EINVAL;
    std::string out;
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        for (const auto& kv : g_tuned) {
            const WalkVariant& w = kVariants[kv.second];
            out += "dev" + std::to_string(kv.first.first) + " groups~2^" + std::to_string(kv.first.second) +
                   ": minblocks " + std::to_string(w.minb) + " bucket " + std::to_string(w.bkt) + "; ";
        }
    }
    out += jt_cell_tuning_text();
    std::snprintf(buf, len, "%s", out.c_str());
    return JT_OK;
}

namespace {

// ------------------------------------------------------------------ cell walk
// The near field as a cell list: per box a grid of nb^3 cells of side
// L / nb >= r_cut (1e-4 margin), holding both species; every pair inside
// r_cut lies in a cell and its 26 neighbours (nb >= 3, so the 27 are
// distinct and the shifted image is the one within r_cut).  One warp per
// cell: its targets (both species, ~30 at the 2x224^3 density) test every
// candidate of the 27 cells that lies within r_cut of their AABB, in dense
// chunks of 32 where every lane evaluates every candidate with the pair
// force selected by r^2 < r_cut^2 (no per-lane hit loop, no traversal).
// Pairs are exactly those of the tree walk when it accepts no multipole
// (the uniform case); cells whose neighbourhood holds more than
// JT_CELL_KMAX candidates (clustered data) flag their particles for the
// tree walk, which keeps its multipoles there.

struct CellArgs {
    const jt_seg_dev* segs;
    const jt_box_dev* boxes;
    const int64_t* pprefix;
    int nseg, nbox;
    const int64_t* cprefix;       // cells per box (nbox + 1)
    jt_cell_bufs cb;
    int parts;
    float kick_frac;
    unsigned long long* stats;
    unsigned* err;
    const float4* pmacc;          // non-null: PM accelerations of the pass (jt_b_interp)
    int64_t npart;
};

__device__ __forceinline__ int cell_of(float x, float halfL, float inv, int nb)
{
    int c = (int)floorf((x + halfL) * inv);
    return c < 0 ? 0 : (c >= nb ? nb - 1 : c);
}

// cell key and slot of every particle (atomics on the cell counts); boxes
// without a grid flag their particles for the tree walk
__global__ void k_cell_key(CellArgs A, int64_t npart)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npart) return;
    const int g = jt_find(A.pprefix, A.nseg, i);
    const jt_seg_dev& SG = A.segs[g];
    const jt_box_dev& B = A.boxes[SG.box];
    if (B.nb == 0) {
        A.cb.tflag[i] = 1;
        A.cb.ccell[i] = -1;
        // the tree walk of a flagged particle walks both species' trees
        if (B.seg[0] >= 0) A.cb.segflag[B.seg[0]] = 1;
        if (B.seg[1] >= 0) A.cb.segflag[B.seg[1]] = 1;
        return;
    }
    const float4 p = SG.pos[i - A.pprefix[g]];
    const int nb = B.nb;
    const int cx = cell_of(p.x, B.halfL, B.cell_inv, nb), cy = cell_of(p.y, B.halfL, B.cell_inv, nb),
              cz = cell_of(p.z, B.halfL, B.cell_inv, nb);
    const int key = (int)(B.cbase + ((int64_t)cz * nb + cy) * nb + cx);
    // one atomic per distinct cell of the warp (Morton-ordered particles
    // mostly share their lanes' cells); slots follow lane order in a group
    const unsigned peers = __match_any_sync(__activemask(), key);
    const int lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
    unsigned base = 0;
    if (lane == leader) base = (unsigned)atomicAdd(A.cb.ccount + key, __popc(peers));
    base = __shfl_sync(peers, base, leader);
    A.cb.cslot[i] = base + (unsigned)__popc(peers & ((1u << lane) - 1u));
    A.cb.ccell[i] = key;
    A.cb.tflag[i] = 0;
}

// exclusive scan of n counts, 1024 per block: block-local scan and block sums
constexpr int kScanB = 1024;
__device__ __forceinline__ int block_excl_scan(int v, int* wsum, int& total)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
        int t = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        wsum[lane] = t;   // inclusive warp-total prefix
    }
    __syncthreads();
    total = wsum[(blockDim.x >> 5) - 1];
    const int before = w > 0 ? wsum[w - 1] : 0;
    __syncthreads();
    return before + x - v;
}

__global__ void k_scan_local(const int* __restrict__ in, int* __restrict__ out, int64_t n, int* __restrict__ bsum)
{
    __shared__ int wsum[32];
    const int64_t i = (int64_t)blockIdx.x * kScanB + threadIdx.x;
    const int v = i < n ? in[i] : 0;
    int total;
    const int e = block_excl_scan(v, wsum, total);
    if (i < n) out[i] = e;
    if (threadIdx.x == 0) bsum[blockIdx.x] = total;
}

// one block: exclusive scan of the block sums in place (chunks of 1024 with
// a running carry); bsum[nblk] = grand total
__global__ void k_scan_sums(int* __restrict__ bsum, int nblk)
{
    __shared__ int wsum[32];
    int carry = 0;
    for (int base = 0; base < nblk; base += kScanB) {
        const int i = base + threadIdx.x;
        const int v = i < nblk ? bsum[i] : 0;
        int total;
        const int e = block_excl_scan(v, wsum, total);
        if (i < nblk) bsum[i] = carry + e;
        carry += total;
    }
    if (threadIdx.x == 0) bsum[nblk] = carry;
}

__global__ void k_scan_add(int* __restrict__ out, int64_t n, const int* __restrict__ bsum, int nblk)
{
    const int64_t i = (int64_t)blockIdx.x * kScanB + threadIdx.x;
    if (i < n) out[i] += bsum[blockIdx.x];
    if (i == 0) out[n] = bsum[nblk];
}

// particles into cell order: (x, y, z, s m) and (segment, index)
__global__ void k_cell_scatter(CellArgs A, int64_t npart)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npart) return;
    const int key = A.cb.ccell[i];
    if (key < 0) return;
    const int g = jt_find(A.pprefix, A.nseg, i);
    const jt_seg_dev& SG = A.segs[g];
    const jt_box_dev& B = A.boxes[SG.box];
    const int64_t idx = i - A.pprefix[g];
    const float4 p = SG.pos[idx];
    const float sm = SG.species == 0 ? B.mass[0] : -B.mass[1];
    const int dst = A.cb.cstart[key] + (int)A.cb.cslot[i];
    A.cb.cpos[dst] = make_float4(p.x, p.y, p.z, sm);
    A.cb.cid[dst] = make_int2(g, (int)idx);
}

// A cell with more targets than one batch takes them in a spatial order:
// sub-cell Morton code (3 bits per axis) of each target, ranked in shared
// memory, so that each batch of 32 covers a compact part of the cell and
// streams only the candidates its box can reach.  Cells with more than
// kCellSortMax targets keep the list's order.
constexpr int kCellSortMax = 256;

struct CellWarpSmem {
    float4 cand[64];
    int2 nrange[27];              // (first, count) of each neighbour cell
    float4 nshift[27];            // periodic shift of its particles
    int key[kCellSortMax];        // sub-cell code << 8 | target's rank in the list
    int order[kCellSortMax];      // batch position -> target offset in the cell
};

// dense evaluation of candidates [0, cnt) for this lane's target: every pair
// computed, the force selected by r^2 < r_cut^2.  Per pair: y = (r^2 + eps^2)
// c^2 indexes the log table by its float bits and G(y) = a + b y (no
// reciprocal square root, no float-int conversion); the lane accumulates
// q_j G(y) d, which the caller scales by s_i c^3.  The target itself (r = 0,
// d = 0) adds nothing and is counted as a hit, which the caller removes.
// SCR: opposite-species pairs read the box's Yukawa table yt.
// CNT: count the lane's pairs inside the cut (the pair counters; one
// instruction per candidate, off unless the caller asks for them).
// Positions come scaled by c = 1 / (2 r_s), so that y = |d|^2 + ye directly
// (ye = eps^2 c^2) and the pair is inside the cut for y < yc.  No clamp on
// the table index: the caller bounds ye >= 2^-32 and yc < 64, so that every
// y of a lane inside the cut indexes the table ([2^-32, 2^6)); lanes outside
// it load nothing.
template <bool SCR, bool CNT>
__device__ __forceinline__ unsigned cell_chunk(const float4* __restrict__ cand, int cnt, const float4& p, float si,
                                               float yc, float ye, Acc3& a, const float2* __restrict__ yt)
{
    unsigned hits = 0;
#pragma unroll 4
    for (int j = 0; j < cnt; j++) {
        const float4 q = cand[j];
        const float dx = q.x - p.x, dy = q.y - p.y, dz = q.z - p.z;
        const float y = fmaf(dz, dz, fmaf(dy, dy, fmaf(dx, dx, ye)));
        const unsigned k = (__float_as_uint(y) >> 14) - JT_LTAB_BASE;
        const float2* __restrict__ tb = (SCR && si * q.w < 0.0f) ? yt : g_ltab;
        const bool in = y < yc;
        // only lanes inside the cut read the table (a predicated load: the
        // ~3/4 of dense candidates outside it issue no L1 request), and the
        // others' weight is selected to zero (one select instead of zeroing
        // the load's registers)
        float2 ab;
        if (in) ab = __ldg(&tb[k]);
        const float w = in ? q.w * fmaf(ab.y, y, ab.x) : 0.0f;
        if (CNT) hits += in ? 1u : 0u;
        a.x = fmaf(w, dx, a.x);
        a.y = fmaf(w, dy, a.y);
        a.z = fmaf(w, dz, a.z);
    }
    return hits;
}

// One batch of a cell's targets: lane l takes target base + l.  Smaller
// batches (16 or 8 targets, the warp's lanes split into 2 or 4 candidate
// streams) test 19 % or 37 % fewer candidates, but each batch streams and
// tests the 27 neighbour cells again: measured 5 % and 33 % slower at
// 2x224^3.  (Two targets per lane for cells with more than 32, which streams
// and tests their candidates once instead of twice, measured slower too: its
// registers lowered the occupancy of the whole kernel.)
// base: the batch's first position in the cell's target order; t0, t1: the
// cell's range of the cell list; sorted: the order comes from S.order
template <int ORDER, int NG, bool SCR, bool CNT>
__device__ __forceinline__ void cell_batch(const CellArgs& A, const jt_box_dev& B, CellWarpSmem& S, int base,
                                           int t0, int t1, bool sorted, int lane, unsigned& pairs,
                                           unsigned& cands)
{
    const unsigned lt = (1u << lane) - 1u;
    // the table covers y in [2^-32, 2^6): a softening below 2^-16 (2 r_s)
    // is raised to it, and the cut is bounded by y < 64 (16 r_s without
    // softening), where the split factor is below 1e-27: the table's last
    // entry, zero, held every y past it
    const float cc = B.c, c2 = cc * cc, ye = fmaxf(B.eps2 * c2, 2.3283064365386963e-10f);
    const float yc = fminf(fmaf(B.rc2, c2, ye), 64.0f * 0.99999f);
    const float slack = B.halfL * 9.5367431640625e-7f, rc2_keep = B.rc2 * 1.00001f;
    const float2* __restrict__ yt = (SCR && B.ytab) ? B.ytab : g_ltab;
    const int pos_in_cell = base + lane;
    const bool valid = t0 + pos_in_cell < t1;
    const int t = t0 + (valid ? (sorted ? S.order[pos_in_cell] : pos_in_cell) : (sorted ? S.order[base] : base));
    const float4 p = A.cb.cpos[t];
    const int2 id = A.cb.cid[t];
    const float si = p.w > 0.f ? 1.0f : -1.0f;
    const float lox = warp_min(p.x), loy = warp_min(p.y), loz = warp_min(p.z);
    const float hix = warp_max(p.x), hiy = warp_max(p.y), hiz = warp_max(p.z);
    const float gcx = 0.5f * (lox + hix), gcy = 0.5f * (loy + hiy), gcz = 0.5f * (loz + hiz);
    const float ghx = 0.5f * (hix - lox) + slack, ghy = 0.5f * (hiy - loy) + slack,
                ghz = 0.5f * (hiz - loz) + slack;
    Acc3 near = {0.f, 0.f, 0.f};
    if (A.parts & 2) {
        const float4 ps = make_float4(p.x * cc, p.y * cc, p.z * cc, p.w);
        unsigned hits = 0;
        int nc = 0;
        for (int nbr = 0; nbr < 27; nbr++) {
            const int2 r = S.nrange[nbr];
            const float4 sh = S.nshift[nbr];
            for (int o = 0; o < r.y; o += 32) {
                bool keep = false;
                float4 c = make_float4(0.f, 0.f, 0.f, 0.f);
                if (o + lane < r.y) {
                    c = A.cb.cpos[r.x + o + lane];
                    c.x += sh.x;
                    c.y += sh.y;
                    c.z += sh.z;
                    const float gx = gap1(c.x - gcx, ghx), gy = gap1(c.y - gcy, ghy), gz = gap1(c.z - gcz, ghz);
                    keep = gx * gx + gy * gy + gz * gz <= rc2_keep;
                }
                const unsigned km = __ballot_sync(0xffffffffu, keep);
                if (keep) S.cand[nc + __popc(km & lt)] = make_float4(c.x * cc, c.y * cc, c.z * cc, c.w);
                nc += __popc(km);
                __syncwarp();
                if (nc >= 32) {
                    hits += cell_chunk<SCR, CNT>(S.cand, 32, ps, si, yc, ye, near, yt);
                    cands += 32;
                    __syncwarp();
                    const float4 t2 = S.cand[32 + lane];
                    __syncwarp();
                    if (lane < nc - 32) S.cand[lane] = t2;
                    nc -= 32;
                    __syncwarp();
                }
            }
        }
        if (nc > 0) {
            hits += cell_chunk<SCR, CNT>(S.cand, nc, ps, si, yc, ye, near, yt);
            cands += nc;
        }
        __syncwarp();
        // the target met itself once (r = 0 < r_cut); an empty slot counts nothing
        if (CNT && valid) pairs += hits - 1u;
        const float sc = si * c2;   // positions scaled by c: sum w (c d)
        near.x *= sc;
        near.y *= sc;
        near.z *= sc;
    }
    if (valid) {
        Acc3 pm = {0.f, 0.f, 0.f};
        if (A.parts & 1)
            pm = A.pmacc ? pm_from_tiles<NG>(A.pmacc, A.npart, A.pprefix[id.x] + id.y) : pm_interp<ORDER, NG>(B, p);
        const jt_seg_dev& SG = A.segs[id.x];
        float ax = si * pm.x + near.x, ay = si * pm.y + near.y, az = si * pm.z + near.z;
        if (SCR && B.force_s && (A.parts & 1)) {
            const Acc3 ps = pm_interp<ORDER, NG, true>(B, p);
            ax += ps.x;
            ay += ps.y;
            az += ps.z;
        }
        SG.acc[id.y] = make_float4(ax, ay, az, 0.f);
        if (A.kick_frac != 0.0f) {
            // as k_walk_acc: the closing half kick, and with kick_frac 1.0
            // the next step's opening half kick after it
            const float drag = B.kick_drag, h = 0.5f * B.dt;
            float4 v = SG.vel[id.y];
            v.x += (ax - drag * v.x) * h;
            v.y += (ay - drag * v.y) * h;
            v.z += (az - drag * v.z) * h;
            if (A.kick_frac > 0.75f) {
                v.x += (ax - drag * v.x) * h;
                v.y += (ay - drag * v.y) * h;
                v.z += (az - drag * v.z) * h;
            }
            SG.vel[id.y] = v;
        }
    }
}

#ifndef JT_CELL_MINB
#define JT_CELL_MINB 6
#endif
template <int ORDER, int NG, bool SCR, bool CNT>
__global__ void __launch_bounds__(kWarps * 32, JT_CELL_MINB) k_walk_cell(CellArgs A, int64_t ncells)
{
    __shared__ CellWarpSmem smem_all[kWarps];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    CellWarpSmem& S = smem_all[wib];
    const int64_t gc = (int64_t)blockIdx.x * kWarps + wib;
    if (gc >= ncells) return;   // whole warp
    const int t0 = A.cb.cstart[gc], t1 = A.cb.cstart[gc + 1];
    if (t0 == t1) return;
    const int k = jt_find(A.cprefix, A.nbox, gc);
    const jt_box_dev& B = A.boxes[k];
    const int nb = B.nb;
    const int64_t local = gc - A.cprefix[k];
    const int cx = (int)(local % nb), cy = (int)((local / nb) % nb), cz = (int)(local / ((int64_t)nb * nb));
    // the 27 neighbour cells: lane l < 27 takes offset (l % 3 - 1, l / 3 % 3 - 1, l / 9 - 1)
    int cnt = 0;
    if (lane < 27) {
        int nx = cx + lane % 3 - 1, ny = cy + (lane / 3) % 3 - 1, nz = cz + lane / 9 - 1;
        float sx = 0.f, sy = 0.f, sz = 0.f;
        if (nx < 0) { nx += nb; sx = -B.L; } else if (nx >= nb) { nx -= nb; sx = B.L; }
        if (ny < 0) { ny += nb; sy = -B.L; } else if (ny >= nb) { ny -= nb; sy = B.L; }
        if (nz < 0) { nz += nb; sz = -B.L; } else if (nz >= nb) { nz -= nb; sz = B.L; }
        const int64_t key = B.cbase + ((int64_t)nz * nb + ny) * nb + nx;
        const int first = A.cb.cstart[key];
        cnt = A.cb.cstart[key + 1] - first;
        S.nrange[lane] = make_int2(first, cnt);
        S.nshift[lane] = make_float4(sx, sy, sz, 0.f);
    }
    int tot = cnt;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
    if (tot > B.cell_kmax) {   // clustered: the tree walk takes these targets
        for (int t = t0 + lane; t < t1; t += 32) {
            const int2 id = A.cb.cid[t];
            A.cb.tflag[A.pprefix[id.x] + id.y] = 1;
        }
        // the tree walk of a flagged particle walks both species' trees
        if (lane == 0 && B.seg[0] >= 0) A.cb.segflag[B.seg[0]] = 1;
        if (lane == 0 && B.seg[1] >= 0) A.cb.segflag[B.seg[1]] = 1;
        return;
    }
    __syncwarp();
    // more than one batch: rank the targets by sub-cell code (3 bits per
    // axis, Morton order) so that consecutive batches are compact
    const int nt = t1 - t0;
    const bool sorted = nt > 32 && nt <= kCellSortMax;
    if (sorted) {
        const float cs = B.L / (float)nb;
        const float ox = (float)cx * cs - B.halfL, oy = (float)cy * cs - B.halfL, oz = (float)cz * cs - B.halfL;
        const float sc = 8.0f / cs;
        for (int i = lane; i < nt; i += 32) {
            const float4 q = A.cb.cpos[t0 + i];
            const int ux = min(max((int)((q.x - ox) * sc), 0), 7), uy = min(max((int)((q.y - oy) * sc), 0), 7),
                      uz = min(max((int)((q.z - oz) * sc), 0), 7);
            int code = 0;
#pragma unroll
            for (int b = 0; b < 3; b++)
                code |= (((ux >> b) & 1) << (3 * b)) | (((uy >> b) & 1) << (3 * b + 1)) | (((uz >> b) & 1) << (3 * b + 2));
            S.key[i] = (code << 8) | i;   // unique: ties by list order
        }
        __syncwarp();
        for (int i = lane; i < nt; i += 32) {
            const int ki = S.key[i];
            int rank = 0;
            for (int j = 0; j < nt; j++) rank += S.key[j] < ki ? 1 : 0;
            S.order[rank] = i;
        }
        __syncwarp();
    }
    unsigned pairs = 0, cands = 0;
    for (int base = 0; base < nt; base += 32)
        cell_batch<ORDER, NG, SCR, CNT>(A, B, S, base, t0, t1, sorted, lane, pairs, cands);
    if (A.stats) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) pairs += __shfl_xor_sync(0xffffffffu, pairs, o);
        if (lane == 0) {
            atomicAdd(A.stats, (unsigned long long)pairs);
            atomicAdd(A.stats + 2, (unsigned long long)cands * 32ull);
        }
    }
}

}  // namespace

int jt_cell_scan_blocks(int64_t ncells) { return (int)((ncells + kScanB - 1) / kScanB); }

int jt_b_cells(const jt_seg_dev* d_segs, const jt_box_dev* d_boxes, const int64_t* d_pprefix, int nseg,
               int64_t npart, const int64_t* d_cprefix, int nbox, int64_t ncells, const jt_cell_bufs& cb,
               int order, int ngrid, int parts, float kick_frac, unsigned long long* stats,
               unsigned* d_err, cudaStream_t st, cudaEvent_t ev_walk0, cudaEvent_t ev_walk1, bool screened,
               const float4* pmacc, bool count_pairs)
{
    cudaEventRecord(ev_walk0, st);   // both recorded on every path (no stale events)
    if (npart <= 0) {
        cudaEventRecord(ev_walk1, st);
        return JT_OK;
    }
    if (int r = stab_ready()) return r;
    CellArgs A;
    A.segs = d_segs;
    A.boxes = d_boxes;
    A.pprefix = d_pprefix;
    A.nseg = nseg;
    A.nbox = nbox;
    A.cprefix = d_cprefix;
    A.cb = cb;
    A.parts = parts;
    A.kick_frac = kick_frac;
    A.stats = stats;
    A.err = d_err;
    A.pmacc = pmacc;
    A.npart = npart;
    const unsigned gp = (unsigned)((npart + 255) / 256);
    if (ncells > 0 && cudaMemsetAsync(cb.ccount, 0, sizeof(int) * (size_t)ncells, st) != cudaSuccess)
        return JT_ECUDA;
    if (cudaMemsetAsync(cb.segflag, 0, sizeof(int) * (size_t)nseg, st) != cudaSuccess) return JT_ECUDA;
    k_cell_key<<<gp, 256, 0, st>>>(A, npart);
    if (ncells == 0) cudaEventRecord(ev_walk1, st);
    if (ncells > 0) {
        const int nblk = jt_cell_scan_blocks(ncells);
        k_scan_local<<<nblk, kScanB, 0, st>>>(cb.ccount, cb.cstart, ncells, cb.bsum);
        k_scan_sums<<<1, kScanB, 0, st>>>(cb.bsum, nblk);
        k_scan_add<<<nblk, kScanB, 0, st>>>(cb.cstart, ncells, cb.bsum, nblk);
        k_cell_scatter<<<gp, 256, 0, st>>>(A, npart);
        const unsigned gw = (unsigned)((ncells + kWarps - 1) / kWarps);
        cudaEventRecord(ev_walk0, st);
#define JT_CELL_LAUNCH(O, N)                                                                    \
    do {                                                                                        \
        if (screened && count_pairs) k_walk_cell<O, N, true, true><<<gw, kWarps * 32, 0, st>>>(A, ncells);   \
        else if (screened) k_walk_cell<O, N, true, false><<<gw, kWarps * 32, 0, st>>>(A, ncells);            \
        else if (count_pairs) k_walk_cell<O, N, false, true><<<gw, kWarps * 32, 0, st>>>(A, ncells);         \
        else k_walk_cell<O, N, false, false><<<gw, kWarps * 32, 0, st>>>(A, ncells);                         \
    } while (0)
        if (order == 4 && ngrid == 2) JT_CELL_LAUNCH(4, 2);
        else if (order == 4 && ngrid == 1) JT_CELL_LAUNCH(4, 1);
        else if (order == 3 && ngrid == 2) JT_CELL_LAUNCH(3, 2);
        else if (order == 3 && ngrid == 1) JT_CELL_LAUNCH(3, 1);
        else if (order == 2 && ngrid == 2) JT_CELL_LAUNCH(2, 2);
        else if (order == 2 && ngrid == 1) JT_CELL_LAUNCH(2, 1);
        else return JT_EINVAL;
#undef JT_CELL_LAUNCH
        cudaEventRecord(ev_walk1, st);
    }
    return cudaGetLastError() == cudaSuccess ? JT_OK : JT_ECUDA;
}

int jt_b_walk(const jt_seg_dev* d_segs, const jt_box_dev* d_boxes, const int64_t* d_gprefix, int nseg,
              int64_t ngroups, const jt_tree_dev& pool, int order, int ngrid, int parts,
              float kick_frac, unsigned long long* stats, unsigned* d_err, cudaStream_t st,
              const int64_t* d_pprefix, const unsigned char* tflag, bool screened, const int* segflag,
              const float4* pmacc, int64_t npart)
{
    if (ngroups <= 0) return JT_OK;
    if (int r = stab_ready()) return r;
    WalkArgs A;
    A.pmacc = pmacc;
    A.npart = npart;
    A.segs = d_segs;
    A.boxes = d_boxes;
    A.gprefix = d_gprefix;
    A.nseg = nseg;
    A.parts = parts;
    A.kick_frac = kick_frac;
    A.pool = pool;
    A.stats = stats;
    A.err = d_err;
    A.pprefix = d_pprefix;
    A.tflag = tflag;
    A.segflag = tflag ? segflag : nullptr;
    unsigned g = (unsigned)((ngroups + kWarps - 1) / kWarps);
    if (screened) {
        if (order == 4 && ngrid == 2) k_walk_acc<4, 2, 6, 32, true><<<g, kWarps * 32, 0, st>>>(A);
        else if (order == 4 && ngrid == 1) k_walk_acc<4, 1, 6, 32, true><<<g, kWarps * 32, 0, st>>>(A);
        else if (order == 3 && ngrid == 2) k_walk_acc<3, 2, 6, 32, true><<<g, kWarps * 32, 0, st>>>(A);
        else if (order == 3 && ngrid == 1) k_walk_acc<3, 1, 6, 32, true><<<g, kWarps * 32, 0, st>>>(A);
        else if (order == 2 && ngrid == 2) k_walk_acc<2, 2, 6, 32, true><<<g, kWarps * 32, 0, st>>>(A);
        else if (order == 2 && ngrid == 1) k_walk_acc<2, 1, 6, 32, true><<<g, kWarps * 32, 0, st>>>(A);
        else return JT_EINVAL;
    } else if (order == 4 && ngrid == 2) launch_variant(pick_variant(g, ngroups, A, st), g, A, st);
    else if (order == 4 && ngrid == 1) k_walk_acc<4, 1, 6, 32, false><<<g, kWarps * 32, 0, st>>>(A);
    else if (order == 3 && ngrid == 2) k_walk_acc<3, 2, 6, 32, false><<<g, kWarps * 32, 0, st>>>(A);
    else if (order == 3 && ngrid == 1) k_walk_acc<3, 1, 6, 32, false><<<g, kWarps * 32, 0, st>>>(A);
    else if (order == 2 && ngrid == 2) k_walk_acc<2, 2, 6, 32, false><<<g, kWarps * 32, 0, st>>>(A);
    else if (order == 2 && ngrid == 1) k_walk_acc<2, 1, 6, 32, false><<<g, kWarps * 32, 0, st>>>(A);
    else return JT_EINVAL;
    return cudaGetLastError() == cudaSuccess ? JT_OK : JT_ECUDA;
}

void jt_launch_walk_rcompat(const jt_rc_params& p, const float4* pos_caller, const int8_t* sign_caller,
                            int64_t n_all, const float4* const spos[2], const int64_t n[2],
                            const jt_tree_dev tree[2], const float* phi, float4* acc_caller,
                            unsigned* d_err, cudaStream_t st)
{
    (void)spos;
    RcArgs A;
    A.p = p;
    A.pos = pos_caller;
    A.sg = sign_caller;
    A.n_all = n_all;
    for (int s = 0; s < 2; s++) {
        A.n[s] = n[s];
        A.tree[s] = tree[s];
    }
    A.phi = phi;
    A.acc = acc_caller;
    A.err = d_err;
    int64_t warps = (n_all + 31) / 32;
    if (warps == 0) return;
    k_walk_rc<<<(unsigned)((warps + kWarps - 1) / kWarps), kWarps * 32, 0, st>>>(A);
}

void jt_launch_kick(float4* vel, const float4* acc, int64_t n, float dt, float drag, cudaStream_t st)
{
    if (n <= 0) return;
    k_kick<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(vel, acc, n, dt, drag);
}

void jt_launch_drift(float4* pos, const float4* vel, int64_t n, float dt, float L, float halfL,
                     cudaStream_t st)
{
    if (n <= 0) return;
    k_drift<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(pos, vel, n, dt, L, halfL);
}

void jt_launch_to_caller(const float4* src, const int* id, const int* gmap, int64_t n, float4* dst,
                         cudaStream_t st)
{
    if (n <= 0) return;
    k_to_caller<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(src, id, gmap, n, dst);
}

void jt_launch_aos_out(const float4* src, const int* id, const int* gmap, int64_t n, float* dst_aos,
                       cudaStream_t st)
{
    if (n <= 0) return;
    k_aos_out<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(src, id, gmap, n, dst_aos);
}

void jt_launch_from_caller(const float4* src_caller, const int* id, const int* gmap, int64_t n,
                           float4* dst, cudaStream_t st)
{
    if (n <= 0) return;
    k_from_caller<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(src_caller, id, gmap, n, dst);
}

void jt_launch_aos_in(const float* src_aos, int64_t n, float4* dst, int* id, cudaStream_t st)
{
    if (n <= 0) return;
    k_aos_in<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(src_aos, n, dst, id);
}

void jt_launch_host_in(const float* src_aos, int64_t n, float4* dst, int* id, cudaStream_t st)
{
    if (n <= 0) return;
    k_host_in<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(src_aos, n, dst, id);
}

void jt_launch_inverse(const int* id, int64_t n, int* inv, cudaStream_t st)
{
    if (n <= 0) return;
    k_inverse<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(id, n, inv);
}

void jt_launch_host_out(const float4* src, const int* inv, int64_t n, float* dst_aos, cudaStream_t st)
{
    if (n <= 0) return;
    k_host_out<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(src, inv, n, dst_aos);
}

void jt_launch_split_signed(const float* pos_aos, const float* vel_aos, const int8_t* sg, int64_t n,
                            const int* rank, float4* pos_p, float4* vel_p, int* id_p, int* gmap_p,
                            float4* pos_m, float4* vel_m, int* id_m, int* gmap_m, cudaStream_t st)
{
    if (n <= 0) return;
    k_split_signed<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(pos_aos, vel_aos, sg, n, rank, pos_p,
                                                                vel_p, id_p, gmap_p, pos_m, vel_m,
                                                                id_m, gmap_m);
}

// ------------------------------------------------------------------ FP32 peak probe
// Independent FMA chains (8 per thread) with no memory traffic: the FP32
// roofline denominator of the walk, measured on the device it runs on.
namespace {
__global__ void k_fma_peak(float* out, int iters, float a, float b)
{
    float x0 = threadIdx.x * 1e-3f, x1 = x0 + 1.f, x2 = x0 + 2.f, x3 = x0 + 3.f;
    float x4 = x0 + 4.f, x5 = x0 + 5.f, x6 = x0 + 6.f, x7 = x0 + 7.f;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int u = 0; u < 16; u++) {
            x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
            x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
        }
    }
    float s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == 1.2345f) out[0] = s;  // keeps the chains alive
}
}  // namespace

extern "C" int jt_fp32_peak(int iters, double* tflops)
{
    if (!tflops || iters <= 0) return JT_EINVAL;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return JT_ECUDA;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    float* out = nullptr;
    if (cudaMalloc(&out, sizeof(float)) != cudaSuccess) return JT_ENOMEM;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    dim3 grid(sms * 8), block(256);
    k_fma_peak<<<grid, block>>>(out, 16, 0.9999f, 1e-4f);  // warm-up
    cudaEventRecord(e0);
    k_fma_peak<<<grid, block>>>(out, iters, 0.9999f, 1e-4f);
    cudaEventRecord(e1);
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (err != cudaSuccess || ms <= 0.f) return JT_ECUDA;
    double flops = 2.0 * 8.0 * 16.0 * (double)iters * grid.x * block.x;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return JT_OK;
}

// ------------------------------------------------------------------ batched step kernels
namespace {

// v += (a - drag_b v) dt over every segment's particles (drag per box)
// the opening kick of kfrac dt followed by the drift of dfrac dt (below), in
// one pass over the particles
__global__ void k_b_kick_drift(const jt_seg_dev* __restrict__ segs, const jt_box_dev* __restrict__ boxes,
                               const int64_t* __restrict__ prefix, int nseg, float kfrac, float dfrac)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= prefix[nseg]) return;
    const int g = jt_find(prefix, nseg, i);
    const int64_t j = i - prefix[g];
    const jt_seg_dev& S = segs[g];
    const jt_box_dev& B = boxes[S.box];
    const float drag = B.kick_drag, dk = kfrac * B.dt, dd = dfrac * B.dt;
    float4 v = S.vel[j], a = S.acc[j], p = S.pos[j];
    v.x += (a.x - drag * v.x) * dk;
    v.y += (a.y - drag * v.y) * dk;
    v.z += (a.z - drag * v.z) * dk;
    S.vel[j] = v;
    p.x += v.x * dd;
    p.y += v.y * dd;
    p.z += v.z * dd;
    p.x = p.x > B.halfL ? p.x - B.L : p.x;
    p.x = p.x < -B.halfL ? p.x + B.L : p.x;
    p.y = p.y > B.halfL ? p.y - B.L : p.y;
    p.y = p.y < -B.halfL ? p.y + B.L : p.y;
    p.z = p.z > B.halfL ? p.z - B.L : p.z;
    p.z = p.z < -B.halfL ? p.z + B.L : p.z;
    S.pos[j] = p;
}

// x += v dt with one periodic wrap per axis (box side per box)
__global__ void k_b_drift(const jt_seg_dev* __restrict__ segs, const jt_box_dev* __restrict__ boxes,
                          const int64_t* __restrict__ prefix, int nseg, float frac)
{
    int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= prefix[nseg]) return;
    const int g = jt_find(prefix, nseg, i);
    const int64_t j = i - prefix[g];
    const jt_seg_dev& S = segs[g];
    const float L = boxes[S.box].L, halfL = boxes[S.box].halfL, dt = frac * boxes[S.box].dt;
    float4 p = S.pos[j], v = S.vel[j];
    p.x += v.x * dt;
    p.y += v.y * dt;
    p.z += v.z * dt;
    p.x = p.x > halfL ? p.x - L : p.x;
    p.x = p.x < -halfL ? p.x + L : p.x;
    p.y = p.y > halfL ? p.y - L : p.y;
    p.y = p.y < -halfL ? p.y + L : p.y;
    p.z = p.z > halfL ? p.z - L : p.z;
    p.z = p.z < -halfL ? p.z + L : p.z;
    S.pos[j] = p;
}

}  // namespace

void jt_b_kick_drift(const jt_seg_dev* d_segs, const jt_box_dev* d_boxes, const int64_t* d_prefix, int nseg,
                     int64_t ntotal, float kfrac, float dfrac, cudaStream_t st)
{
    if (ntotal <= 0) return;
    k_b_kick_drift<<<(unsigned)((ntotal + 255) / 256), 256, 0, st>>>(d_segs, d_boxes, d_prefix, nseg, kfrac,
                                                                      dfrac);
}

void jt_b_drift(const jt_seg_dev* d_segs, const jt_box_dev* d_boxes, const int64_t* d_prefix, int nseg,
                int64_t ntotal, float frac, cudaStream_t st)
{
    if (ntotal <= 0) return;
    k_b_drift<<<(unsigned)((ntotal + 255) / 256), 256, 0, st>>>(d_segs, d_boxes, d_prefix, nseg, frac);
}

namespace {

// S_Y(x; b), x = r_p / (2 r_s), b = kappa r_s, as a function of y = x^2:
// r_p^2 times the force of the short part of the Yukawa split,
// (1 / 2r) [e^{-kr} erfc(x - b) + e^{kr} erfc(x + b)] with kr = 2 b x:
//   S_Y = (Em Cm + Ep Cp) / 2 + b x (Em Cm - Ep Cp) + (2x / sqrt(pi)) e^{-x^2 - b^2},
//   Em = e^{-2bx}, Cm = erfc(x - b), Ep = e^{2bx}, Cp = erfc(x + b);
// b = 0 gives erfc(x) + (2x / sqrt(pi)) e^{-x^2}.  Ep Cp = e^{-x^2 - b^2}
// erfcx(x + b) is taken from its asymptotic series where erfc underflows.
double yukawa_S(double b, double y)
{
    const double x = std::sqrt(y);
    const double em = std::exp(-2.0 * b * x), cm = std::erfc(x - b);
    const double u = x + b;
    double epcp;
    if (u < 25.0) {
        epcp = std::exp(2.0 * b * x) * std::erfc(u);
    } else {
        const double iu2 = 1.0 / (u * u);
        epcp = std::exp(-x * x - b * b) / (u * 1.7724538509055159) * (1.0 - 0.5 * iu2 + 0.75 * iu2 * iu2);
    }
    return 0.5 * (em * cm + epcp) + b * x * (em * cm - epcp) + 1.1283791670955126 * x * std::exp(-x * x - b * b);
}

}  // namespace

void jt_yukawa_log_table(double b, float2* tab)
{
    fill_log_table([b](double y) { return yukawa_S(b, y); }, tab);
}

