// C ABI of the engine: handle, state, force and step pipelines.
//
// One handle = one simulation box on the current device with its own stream,
// cuFFT plans and buffers (the reference keeps process-global cuFFT plans and
// k-space buffers, cuda/cufft_wrapper.cu:30-32, 319-320, and synchronises the
// device after every launch; here nothing is global and a call synchronises
// its own stream once, at the end).
//
// JT_ACCURATE handles are a batch of one box (jt_batch.cu): the same
// one-launch-per-stage pipeline that advances ensembles, so a single box and a
// box inside a batch run identical kernels.  JT_RCOMPAT handles keep the
// reference's caller-order, 64-bit-key formulation here:
//   per species: Morton keys (m30 << 32 | index) -> onesweep sort -> reorder
//   -> Karras nodes -> cube moments;  memset rho -> CIC deposit in caller
//   order -> R2C -> Green's function -> C2R (potential);  warp-uniform walk
//   with finite-difference PM gradient.
#include "jt_batch.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <map>
#include <mutex>
#include <new>
#include <utility>
#include <vector>

int jt_smem_attr(const void* kernel, int bytes)
{
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, int> done;   // (device, kernel) -> bytes set
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return JT_ECUDA;
    std::lock_guard<std::mutex> lock(mu);
    int& have = done[std::make_pair(dev, kernel)];
    if (have >= bytes) return JT_OK;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) != cudaSuccess)
        return JT_ECUDA;
    have = bytes;
    return JT_OK;
}

struct jt_handle {
    jt_config cfg;
    int device = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t ev[10] = {};
    int64_t n[2] = {0, 0};
    float mass[2] = {0.f, 0.f};
    bool have_state = false;
    bool signed_layout = false;
    bool acc_valid = false;
    int64_t cap[2] = {0, 0};
    float4 *pos[2] = {}, *vel[2] = {}, *acc[2] = {}, *pos_b[2] = {}, *vel_b[2] = {};
    int *id[2] = {}, *id_b[2] = {}, *gmap[2] = {};
    jt_tree_dev tree[2] = {};
    jt_sort_ws ws = {};
    uint64_t* key64 = nullptr;
    jt_pm_dev pm = {};
    float4* pos_caller = nullptr;
    float4* acc_caller = nullptr;
    int8_t* sign_caller = nullptr;
    int* rank_buf = nullptr;
    void* stage = nullptr;
    size_t stage_bytes = 0;
    unsigned* d_err = nullptr;
    unsigned long long* d_stats = nullptr;   // pairs, nodes, candidates
    jt_timings tm = {};
    int64_t phase[4] = {0, 0, 0, 0};   // walk phase counters of a diagnostic build
    // JT_ACCURATE: the particle state lives in box `box_id` of `batch`
    jt_batch* batch = nullptr;
    int box_id = -1;
    bool dbg_ready = false;            // debug-tree buffers (accurate mode)
    // Yukawa screening of opposite-sign pairs: lambda_0 > 0.01 selects the
    // screened walk (compatibility mode) or the screened split (accurate
    // mode, applied to the handle's batch box)
    double lambda_0 = 0.0, z = 0.0;
};

namespace {

// The particle arrays of a handle (internal order).  In accurate mode they
// belong to the batch box and change after every force pass (the reorder
// swaps buffers), so take a fresh view after each pass.
struct Parts {
    float4* pos[2];
    float4* vel[2];
    float4* acc[2];
    int* id[2];
};

Parts parts_of(jt_handle* h)
{
    Parts p;
    jt_box_state* b = h->batch ? jtb_box(h->batch, h->box_id) : nullptr;
    for (int s = 0; s < 2; s++) {
        p.pos[s] = b ? b->pos[s] : h->pos[s];
        p.vel[s] = b ? b->vel[s] : h->vel[s];
        p.acc[s] = b ? b->acc[s] : h->acc[s];
        p.id[s] = b ? b->id[s] : h->id[s];
    }
    return p;
}

}  // namespace

namespace {

bool cuda_ok(cudaError_t e) { return e == cudaSuccess; }

#define JT_TRY(x)                      \
    do {                               \
        int _r = (x);                  \
        if (_r != JT_OK) return _r;    \
    } while (0)
#define JT_CU(x)                                   \
    do {                                           \
        if ((x) != cudaSuccess) return JT_ECUDA;   \
    } while (0)
#define JT_FFT(x)                                   \
    do {                                            \
        if ((x) != CUFFT_SUCCESS) return JT_ECUDA;  \
    } while (0)

template <class T>
int dalloc(T** p, size_t count)
{
    *p = nullptr;
    if (count == 0) count = 1;
    return cuda_ok(cudaMalloc((void**)p, sizeof(T) * count)) ? JT_OK : JT_ENOMEM;
}

template <class T>
void dfree(T*& p)
{
    if (p) cudaFree((void*)p);
    p = nullptr;
}

bool is_pow2(int m) { return m > 0 && (m & (m - 1)) == 0; }

int validate(const jt_config* c)
{
    if (!c) return JT_EINVAL;
    if (!(c->box_L > 0.0) || !std::isfinite(c->box_L)) return JT_EINVAL;
    if (!is_pow2(c->pm_grid) || c->pm_grid < 8 || c->pm_grid > 1024) return JT_EINVAL;
    if (!(c->theta >= 0.0) || !std::isfinite(c->theta)) return JT_EINVAL;
    if (!(c->softening >= 0.0) || !std::isfinite(c->softening)) return JT_EINVAL;
    if (!(c->r_cut > 0.0) || c->r_cut >= 0.5 * c->box_L) return JT_EINVAL;
    if (c->mode == JT_ACCURATE && !(c->r_s > 0.0)) return JT_EINVAL;
    if (c->cut_tail_ppm < 0 || c->cut_tail_ppm >= 1000000) return JT_EINVAL;
    if (c->mode == JT_ACCURATE && !(jt_short_cut(*c) < 0.5 * c->box_L)) return JT_EINVAL;
    if (!(c->mu >= 0.0) || !std::isfinite(c->mu)) return JT_EINVAL;
    if (!(c->G_mass_plus > 0.0) || !std::isfinite(c->G_mass_plus)) return JT_EINVAL;
    if (c->k_min < 0) return JT_EINVAL;
    if (c->mode != JT_ACCURATE && c->mode != JT_RCOMPAT) return JT_EINVAL;
    if (c->integrator != JT_KDK && c->integrator != JT_DKD_REF) return JT_EINVAL;
    if (c->pm_order != 0 && (c->pm_order < 2 || c->pm_order > 4)) return JT_EINVAL;
    if (c->pm_interlace < 0 || c->pm_interlace > 2) return JT_EINVAL;
    return JT_OK;
}

}  // namespace

extern "C" int jt_config_short_cut(const jt_config* cfg, double* cut)
{
    if (!cfg || !cut) return JT_EINVAL;
    if (int r = validate(cfg)) return r;
    *cut = cfg->mode == JT_ACCURATE ? jt_short_cut(*cfg) : cfg->r_cut;
    return JT_OK;
}

namespace {

void free_trees(jt_handle* h)
{
    for (int s = 0; s < 2; s++) {
        jt_tree_dev& t = h->tree[s];
        dfree(t.child); dfree(t.range); dfree(t.parent); dfree(t.flag); dfree(t.com); dfree(t.bmin);
        dfree(t.bmax); dfree(t.quad0); dfree(t.quad1); dfree(t.m30); dfree(t.tie);
        t = jt_tree_dev{};
    }
    jt_sort_ws_free(&h->ws);
    dfree(h->key64);
    h->dbg_ready = false;
}

void free_particles(jt_handle* h)
{
    for (int s = 0; s < 2; s++) {
        dfree(h->pos[s]); dfree(h->vel[s]); dfree(h->acc[s]);
        dfree(h->pos_b[s]); dfree(h->vel_b[s]);
        dfree(h->id[s]); dfree(h->id_b[s]); dfree(h->gmap[s]);
        h->cap[s] = 0;
    }
    free_trees(h);
    if (h->batch && h->box_id >= 0) jt_batch_remove(h->batch, h->box_id);
    h->box_id = -1;
    dfree(h->pos_caller); dfree(h->acc_caller); dfree(h->sign_caller); dfree(h->rank_buf);
    if (h->stage) cudaFree(h->stage);
    h->stage = nullptr;
    h->stage_bytes = 0;
}

// Trees, sort workspace and 64-bit keys for both species (RCOMPAT force
// passes, and jt_debug_tree in either mode).
int alloc_trees(jt_handle* h, int64_t n0, int64_t n1)
{
    int64_t nn[2] = {n0, n1};
    for (int s = 0; s < 2; s++) {
        int64_t n = nn[s], nodes = n > 0 ? 2 * n - 1 : 1;
        jt_tree_dev& t = h->tree[s];
        JT_TRY(dalloc(&t.child, nodes)); JT_TRY(dalloc(&t.parent, nodes));
        JT_TRY(dalloc(&t.range, n > 1 ? n - 1 : 1));
        JT_TRY(dalloc(&t.flag, n > 1 ? n - 1 : 1));
        JT_TRY(dalloc(&t.com, nodes)); JT_TRY(dalloc(&t.bmin, nodes)); JT_TRY(dalloc(&t.bmax, nodes));
        JT_TRY(dalloc(&t.quad0, nodes)); JT_TRY(dalloc(&t.quad1, nodes));
        JT_TRY(dalloc(&t.m30, n)); JT_TRY(dalloc(&t.tie, n));
        t.n = n;
    }
    int64_t nmax = n0 > n1 ? n0 : n1;
    if (jt_sort_ws_alloc(&h->ws, nmax > 0 ? nmax : 1, 8) != 0) return JT_ENOMEM;
    JT_TRY(dalloc(&h->key64, nmax));
    h->dbg_ready = true;
    return JT_OK;
}

int alloc_particles(jt_handle* h, int64_t n0, int64_t n1)
{
    if (h->stage && h->cap[0] == n0 && h->cap[1] == n1) {  // same sizes: reuse
        if (h->batch) {
            jt_box_state* b = jtb_box(h->batch, h->box_id);
            if (b) b->acc_valid = false;
        }
        return JT_OK;
    }
    free_particles(h);
    int64_t nn[2] = {n0, n1};
    for (int s = 0; s < 2; s++) JT_TRY(dalloc(&h->gmap[s], nn[s]));
    if (h->batch) {
        JT_TRY(jtb_add_empty(h->batch, &h->cfg, n0, n1, &h->box_id));
        if (h->lambda_0 > 0.01) JT_TRY(jt_batch_set_screening(h->batch, h->box_id, h->lambda_0, h->z));
    } else {
        for (int s = 0; s < 2; s++) {
            int64_t n = nn[s];
            JT_TRY(dalloc(&h->pos[s], n)); JT_TRY(dalloc(&h->vel[s], n)); JT_TRY(dalloc(&h->acc[s], n));
            JT_TRY(dalloc(&h->pos_b[s], n)); JT_TRY(dalloc(&h->vel_b[s], n));
            JT_TRY(dalloc(&h->id[s], n)); JT_TRY(dalloc(&h->id_b[s], n));
        }
        JT_TRY(alloc_trees(h, n0, n1));
    }
    int64_t na = n0 + n1;
    JT_TRY(dalloc(&h->pos_caller, h->batch ? 1 : na)); JT_TRY(dalloc(&h->acc_caller, h->batch ? 1 : na));
    JT_TRY(dalloc(&h->sign_caller, na)); JT_TRY(dalloc(&h->rank_buf, na));
    h->stage_bytes = sizeof(float) * 3 * (size_t)(na > 0 ? na : 1) * 2;
    if (!cuda_ok(cudaMalloc(&h->stage, h->stage_bytes))) return JT_ENOMEM;
    h->cap[0] = n0;
    h->cap[1] = n1;
    return JT_OK;
}

// RCOMPAT PM: one CIC grid, its spectrum (Green's function applied in
// place) and the potential grid.
int alloc_pm(jt_handle* h)
{
    jt_pm_dev& pm = h->pm;
    const jt_config& c = h->cfg;
    int M = c.pm_grid;
    pm.M = M;
    pm.L = c.box_L;
    pm.order = 2;
    pm.ngrid = 1;
    int64_t G = (int64_t)M * M * M, Gc = (int64_t)M * M * (M / 2 + 1);
    JT_TRY(dalloc(&pm.rho, G));
    JT_TRY(dalloc(&pm.force_k, Gc));
    JT_TRY(dalloc(&pm.force, G));
    JT_FFT(cufftPlan3d(&pm.plan_r2c, M, M, M, CUFFT_R2C));
    if (cufftPlan3d(&pm.plan_c2r, M, M, M, CUFFT_C2R) != CUFFT_SUCCESS) {
        cufftDestroy(pm.plan_r2c);
        return JT_ECUDA;
    }
    pm.plans_ready = 1;
    JT_FFT(cufftSetStream(pm.plan_r2c, h->st));
    JT_FFT(cufftSetStream(pm.plan_c2r, h->st));
    return JT_OK;
}

void free_pm(jt_handle* h)
{
    jt_pm_dev& pm = h->pm;
    if (pm.plans_ready) {
        cufftDestroy(pm.plan_r2c);
        cufftDestroy(pm.plan_c2r);
    }
    dfree(pm.rho); dfree(pm.force_k); dfree(pm.force);
    pm = jt_pm_dev{};
}

int id_bits(int64_t n)
{
    int b = 0;
    while (b < 32 && ((int64_t)1 << b) < n) b++;
    return b;
}

// RCOMPAT: sort both species by the reference's 64-bit Morton key
// (m30 << 32 | caller index), reorder the state, build both trees with the
// reference's cube node geometry.
int build_trees(jt_handle* h)
{
    float box_half = (float)(h->cfg.box_L / 2.0);
    for (int s = 0; s < 2; s++) {
        int64_t n = h->n[s];
        if (n == 0) continue;
        jt_tree_dev& t = h->tree[s];
        jt_launch_morton(h->pos[s], h->id[s], n, box_half, nullptr, h->key64, h->ws.vals, h->st);
        int shifts[8], np = 0;
        int ib = id_bits(n);
        for (int b = 0; b < ib; b += 8) shifts[np++] = b;
        for (int b = 32; b < 62; b += 8) shifts[np++] = b;
        JT_TRY(jt_radix_sort_u64(h->key64, h->ws.vals, n, shifts, np, &h->ws, h->d_err, h->st));
        jt_launch_split_keys(h->key64, n, t.m30, t.tie, h->st);
        jt_launch_reorder(h->ws.vals, n, h->pos[s], h->pos_b[s], h->vel[s], h->vel_b[s], h->id[s],
                          h->id_b[s], h->st);
        std::swap(h->pos[s], h->pos_b[s]);
        std::swap(h->vel[s], h->vel_b[s]);
        std::swap(h->id[s], h->id_b[s]);
        t.n = n;
        h->tm.launches += 5 + np;   // morton, hist, scan, np onesweep passes, split, reorder
    }
    cudaEventRecord(h->ev[1], h->st);
    for (int s = 0; s < 2; s++) {
        int64_t n = h->n[s];
        if (n == 0) continue;
        jt_launch_karras(h->tree[s], h->st);
        jt_launch_moments_rc(h->tree[s], h->pos[s], h->mass[s], box_half, h->st);
        h->tm.launches += (n > 1 ? 1 : 0) + 1;
    }
    return cudaGetLastError() == cudaSuccess ? JT_OK : JT_ECUDA;
}

int check_device_error(jt_handle* h)
{
    unsigned e = 0;
    JT_CU(cudaMemcpyAsync(&e, h->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, h->st));
    JT_CU(cudaStreamSynchronize(h->st));
    if (e) {
        cudaMemsetAsync(h->d_err, 0, sizeof(unsigned), h->st);
        cudaStreamSynchronize(h->st);
        if (e & JT_ERRBIT_LOOKBACK) return JT_ETIMEDOUT;
        return JT_EOVERFLOW;
    }
    return JT_OK;
}

float elapsed(cudaEvent_t a, cudaEvent_t b)
{
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) return 0.f;
    return ms;
}

// RCOMPAT accelerations at the current positions into acc[s] (internal
// order); kick_dt/drag: a kick applied after the walk (0 = none).
int compute_forces_rc(jt_handle* h, float kick_dt, float drag, int parts = JT_PART_ALL)
{
    const jt_config& c = h->cfg;
    cudaStream_t st = h->st;
    int M = c.pm_grid;
    int64_t G = (int64_t)M * M * M;
    cudaEventRecord(h->ev[0], st);
    JT_TRY(build_trees(h));
    cudaEventRecord(h->ev[2], st);
    JT_CU(cudaMemsetAsync(h->pm.rho, 0, sizeof(float) * G, st));
    for (int s = 0; s < 2; s++)
        jt_launch_to_caller(h->pos[s], h->id[s], h->gmap[s], h->n[s], h->pos_caller, st);
    double cell = c.box_L / M;
    jt_launch_rcompat_deposit(h->pos_caller, h->sign_caller, h->n[0] + h->n[1], h->mass, h->pm.rho, M,
                              (float)(c.box_L / 2.0), (float)(M / c.box_L),
                              (float)(1.0 / (cell * cell * cell)), st);
    cudaEventRecord(h->ev[3], st);
    JT_FFT(cufftExecR2C(h->pm.plan_r2c, h->pm.rho, h->pm.force_k));
    cudaEventRecord(h->ev[4], st);
    jt_launch_kspace_rc(h->pm.force_k, M, c.box_L, c.r_cut / 3.0, c.k_min, st);
    cudaEventRecord(h->ev[5], st);
    JT_FFT(cufftExecC2R(h->pm.plan_c2r, h->pm.force_k, h->pm.force));
    cudaEventRecord(h->ev[6], st);
    float tq, sq, rq, bq, il = 0.0f;
    const bool screened = h->lambda_0 > 0.01;
    {
        // host packing of the reference (:4079-4082, :1932-1937) and the
        // kernel's unpacking (:1684-1694); the screened branch rounds theta
        // and softening (:4009-4011) and packs lambda(z) = lambda_0 sqrt(1+z)
        // with box_half (:4015, :1921-1927; unpacked at :929-936, :952)
        auto sat = [](double v) -> unsigned {
            return !(v > 0.0) ? 0u : (v >= 4294967295.0 ? 0xFFFFFFFFu : (unsigned)v);
        };
        const double tv = screened ? std::round(c.theta * 1000.0) : c.theta * 1000.0;
        const double sv = screened ? std::round(c.softening * 1000.0) : c.softening * 1000.0;
        unsigned ti = sat(tv), si = sat(sv);
        unsigned ri = sat(c.r_cut), bi = sat(c.box_L / 2.0);
        unsigned li = sat(h->lambda_0 * std::sqrt(1.0 + h->z) * 10.0);
        ti = ti > 0xFFFF ? 0xFFFF : ti; si = si > 0xFFFF ? 0xFFFF : si;
        ri = ri > 0xFFFF ? 0xFFFF : ri; bi = bi > 0xFFFF ? 0xFFFF : bi;
        li = li > 0xFFFF ? 0xFFFF : li;
        tq = (float)ti / 1000.0f; sq = (float)si / 1000.0f; rq = (float)ri; bq = (float)bi;
        const float lam = (float)li / 10.0f;
        if (screened) il = lam > 0.01f ? 1.0f / lam : 0.0f;
    }
    jt_rc_params P;
    P.theta2 = tq * tq;
    P.eps2 = sq * sq;
    P.r_cut = rq;
    P.box_half_q = bq;
    P.r_s = rq / 3.0f;
    P.box_half = (float)(c.box_L / 2.0);
    P.inv_cell = (float)(M / c.box_L);
    P.cell = (float)(c.box_L / M);
    P.M = M;
    P.mass[0] = h->mass[0];
    P.mass[1] = h->mass[1];
    P.parts = parts;
    P.screen = screened ? 1 : 0;
    P.inv_lambda = il;
    const float4* sp2[2] = {h->pos[0], h->pos[1]};
    jt_launch_walk_rcompat(P, h->pos_caller, h->sign_caller, h->n[0] + h->n[1], sp2, h->n, h->tree,
                           h->pm.force, h->acc_caller, h->d_err, st);
    for (int s = 0; s < 2; s++)
        jt_launch_from_caller(h->acc_caller, h->id[s], h->gmap[s], h->n[s], h->acc[s], st);
    if (kick_dt != 0.0f)
        for (int s = 0; s < 2; s++) jt_launch_kick(h->vel[s], h->acc[s], h->n[s], kick_dt, drag, st);
    cudaEventRecord(h->ev[7], st);
    JT_CU(cudaGetLastError());
    const int nsp = (h->n[0] > 0) + (h->n[1] > 0);
    // to_caller, from_caller (and kick) per species; deposit, k-space, walk
    h->tm.launches += (kick_dt != 0.0f ? 3 : 2) * nsp + 3;
    h->acc_valid = parts == JT_PART_ALL;
    return JT_OK;
}

void accumulate_timings(jt_handle* h)
{
    // ev0 start, ev1 (last species) karras start, ev2 trees done, ev3 deposit
    // done, ev4 R2C done, ev5 k-space done, ev6 C2R done, ev7 walk done
    h->tm.sort_ms += elapsed(h->ev[0], h->ev[1]);
    h->tm.tree_ms += elapsed(h->ev[1], h->ev[2]);
    h->tm.deposit_ms += elapsed(h->ev[2], h->ev[3]);
    h->tm.fft_ms += elapsed(h->ev[3], h->ev[6]);
    h->tm.kspace_ms += elapsed(h->ev[4], h->ev[5]);
    h->tm.walk_ms += elapsed(h->ev[6], h->ev[7]);
}

int fetch_inter(jt_handle* h)
{
    unsigned long long v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    JT_CU(cudaMemcpyAsync(v, h->d_stats, sizeof(v), cudaMemcpyDeviceToHost, h->st));
    JT_CU(cudaStreamSynchronize(h->st));
    h->tm.pair_interactions += (int64_t)v[0];
    h->tm.node_interactions += (int64_t)v[1];
    h->tm.candidates += (int64_t)v[2];
    h->tm.interactions += (int64_t)(v[0] + v[1]);
    for (int i = 0; i < 4; i++) h->phase[i] += (int64_t)v[3 + i];
    JT_CU(cudaMemsetAsync(h->d_stats, 0, sizeof(v), h->st));
    return JT_OK;
}

void set_masses(jt_handle* h)
{
    double mp = h->cfg.G_mass_plus;
    double mm = h->n[1] > 0 ? h->cfg.mu * mp * (double)h->n[0] / (double)h->n[1] : 0.0;
    if (h->n[0] == 0) mm = h->cfg.mu * mp;  // no m+ particles: m- per particle = mu * m+
    h->mass[0] = (float)mp;
    h->mass[1] = (float)mm;
}

__global__ void k_iota(int* __restrict__ dst, int64_t n, int off)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = (int)(off + i);
}

// [m+ ; m-] signs of the per-species layout
__global__ void k_layout_signs(int8_t* __restrict__ dst, int64_t n0, int64_t n)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = i < n0 ? (int8_t)1 : (int8_t)-1;
}

// dst[i] = AoS row id[i] of src (caller order -> internal order)
__global__ void k_aos_gather(const float* __restrict__ src, const int* __restrict__ id, int64_t n,
                             float4* __restrict__ dst)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int64_t k = 3 * (int64_t)id[i];
    dst[i] = make_float4(src[k], src[k + 1], src[k + 2], 0.f);
}

int copy_in(jt_handle* h, const void* src, size_t bytes, int mem, void** dev)
{
    if (mem == JT_MEM_DEVICE) {
        *dev = const_cast<void*>(src);
        return JT_OK;
    }
    if (bytes > h->stage_bytes) return JT_EINVAL;
    JT_CU(cudaMemcpyAsync(h->stage, src, bytes, cudaMemcpyHostToDevice, h->st));
    *dev = h->stage;
    return JT_OK;
}

int write_out(jt_handle* h, const float4* src, const int* id, const int* gmap, int64_t n,
              float* dst, int mem)
{
    if (!dst || n == 0) return JT_OK;
    float* target = mem == JT_MEM_DEVICE ? dst : (float*)h->stage;
    jt_launch_aos_out(src, id, gmap, n, target, h->st);
    if (mem == JT_MEM_HOST)
        JT_CU(cudaMemcpyAsync(dst, h->stage, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, h->st));
    return JT_OK;
}

}  // namespace

extern "C" {

const char* jt_version(void) { return "janus-treepm-b200 0.1 sm_100a"; }

const char* jt_strerror(int code)
{
    switch (code) {
    case JT_OK: return "ok";
    case JT_EINVAL: return "invalid argument";
    case JT_ENOMEM: return "out of memory";
    case JT_ECUDA: return "CUDA or cuFFT error";
    case JT_ETIMEDOUT: return "device wait timed out";
    case JT_ENOTIMPL: return "not implemented";
    case JT_ESTATE: return "call out of order";
    case JT_EOVERFLOW: return "device list overflow";
    case JT_EBUSY: return "admission refused";
    default: return "unknown error";
    }
}

int jt_create(const jt_config* cfg, jt_handle** out)
{
    if (!out) return JT_EINVAL;
    *out = nullptr;
    JT_TRY(validate(cfg));
    jt_handle* h = new (std::nothrow) jt_handle();
    if (!h) return JT_ENOMEM;
    h->cfg = *cfg;
    int r = JT_OK;
    if (cudaGetDevice(&h->device) != cudaSuccess) {
        delete h;
        return JT_ECUDA;
    }
    if (cfg->mode == JT_ACCURATE) {
        // a batch of one box; the handle issues its own launches on the
        // batch's stream so that everything stays in stream order
        r = jt_batch_create(&h->batch);
        if (r != JT_OK) {
            delete h;
            return r;
        }
        h->st = jtb_stream(h->batch);
    } else if (cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking) != cudaSuccess) {
        delete h;
        return JT_ECUDA;
    }
    for (auto& e : h->ev) cudaEventCreate(&e);
    if (cudaMalloc(&h->d_err, sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&h->d_stats, 8 * sizeof(unsigned long long)) != cudaSuccess) r = JT_ENOMEM;
    if (r == JT_OK) {
        cudaMemset(h->d_err, 0, sizeof(unsigned));
        cudaMemset(h->d_stats, 0, 8 * sizeof(unsigned long long));
        if (!h->batch) r = alloc_pm(h);
    }
    if (r != JT_OK) {
        jt_destroy(h);
        return r;
    }
    *out = h;
    return JT_OK;
}

void jt_destroy(jt_handle* h)
{
    if (!h) return;
    if (h->st) cudaStreamSynchronize(h->st);
    free_particles(h);
    free_pm(h);
    if (h->d_err) cudaFree(h->d_err);
    if (h->d_stats) cudaFree(h->d_stats);
    for (auto& e : h->ev)
        if (e) cudaEventDestroy(e);
    if (h->batch) {
        jt_batch_destroy(h->batch);   // owns the stream
    } else if (h->st) {
        cudaStreamDestroy(h->st);
    }
    delete h;
}

int jt_set_state(jt_handle* h, const float* pos_p, const float* vel_p, size_t n_p,
                 const float* pos_m, const float* vel_m, size_t n_m, int mem)
{
    if (!h || (mem != JT_MEM_HOST && mem != JT_MEM_DEVICE)) return JT_EINVAL;
    if ((n_p && !pos_p) || (n_m && !pos_m)) return JT_EINVAL;
    if (n_p + n_m == 0) return JT_EINVAL;
    if (n_p >= (size_t)1 << 30 || n_m >= (size_t)1 << 30) return JT_EINVAL;
    h->have_state = false;
    h->acc_valid = false;
    JT_TRY(alloc_particles(h, (int64_t)n_p, (int64_t)n_m));
    h->n[0] = (int64_t)n_p;
    h->n[1] = (int64_t)n_m;
    set_masses(h);
    const Parts P = parts_of(h);
    const float* pp[2] = {pos_p, pos_m};
    const float* vv[2] = {vel_p, vel_m};
    // host arrays: all copies back to back into disjoint parts of the
    // staging buffer (6 (n+ + n-) floats), then the conversions
    const float* dp[2] = {pos_p, pos_m};
    const float* dv[2] = {vel_p, vel_m};
    if (mem == JT_MEM_HOST) {
        float* st = (float*)h->stage;
        size_t off = 0;
        for (int s = 0; s < 2; s++) {
            const size_t b = sizeof(float) * 3 * (size_t)h->n[s];
            if (h->n[s] == 0) continue;
            JT_CU(cudaMemcpyAsync(st + off, pp[s], b, cudaMemcpyHostToDevice, h->st));
            dp[s] = st + off;
            off += 3 * (size_t)h->n[s];
            if (vv[s]) {
                JT_CU(cudaMemcpyAsync(st + off, vv[s], b, cudaMemcpyHostToDevice, h->st));
                dv[s] = st + off;
                off += 3 * (size_t)h->n[s];
            }
        }
    }
    for (int s = 0; s < 2; s++) {
        const int64_t n = h->n[s];
        if (n == 0) continue;
        jt_launch_aos_in(dp[s], n, P.pos[s], P.id[s], h->st);
        if (vv[s])
            jt_launch_aos_in(dv[s], n, P.vel[s], nullptr, h->st);
        else
            JT_CU(cudaMemsetAsync(P.vel[s], 0, sizeof(float4) * n, h->st));
        // caller layout: [m+ ; m-]
        k_iota<<<(unsigned)((n + 255) / 256), 256, 0, h->st>>>(h->gmap[s], n, s == 1 ? (int)h->n[0] : 0);
    }
    const int64_t na = h->n[0] + h->n[1];
    k_layout_signs<<<(unsigned)((na + 255) / 256), 256, 0, h->st>>>(h->sign_caller, h->n[0], na);
    JT_CU(cudaGetLastError());
    JT_CU(cudaStreamSynchronize(h->st));
    h->tm.launches += 2 * ((h->n[0] > 0) + (h->n[1] > 0)) + 1;
    h->signed_layout = false;
    h->have_state = true;
    return JT_OK;
}

int jt_set_state_signed(jt_handle* h, const float* pos, const float* vel, const int8_t* signs,
                        size_t n, int mem)
{
    if (!h || !pos || !signs || n == 0 || (mem != JT_MEM_HOST && mem != JT_MEM_DEVICE))
        return JT_EINVAL;
    if (n >= (size_t)1 << 30) return JT_EINVAL;
    std::vector<int8_t> sg(n);
    if (mem == JT_MEM_DEVICE) {
        JT_CU(cudaMemcpy(sg.data(), signs, n, cudaMemcpyDeviceToHost));
    } else {
        std::memcpy(sg.data(), signs, n);
    }
    std::vector<int> rank(n);
    int64_t c[2] = {0, 0};
    for (size_t i = 0; i < n; i++) {
        if (sg[i] != 1 && sg[i] != -1) return JT_EINVAL;
        int s = sg[i] > 0 ? 0 : 1;
        rank[i] = (int)c[s]++;
    }
    h->have_state = false;
    h->acc_valid = false;
    JT_TRY(alloc_particles(h, c[0], c[1]));
    h->n[0] = c[0];
    h->n[1] = c[1];
    set_masses(h);
    JT_CU(cudaMemcpyAsync(h->rank_buf, rank.data(), sizeof(int) * n, cudaMemcpyHostToDevice, h->st));
    JT_CU(cudaMemcpyAsync(h->sign_caller, sg.data(), n, cudaMemcpyHostToDevice, h->st));
    const float* dpos = pos;
    const float* dvel = vel;
    if (mem == JT_MEM_HOST) {
        float* stg = (float*)h->stage;
        JT_CU(cudaMemcpyAsync(stg, pos, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, h->st));
        dpos = stg;
        if (vel) {
            JT_CU(cudaMemcpyAsync(stg + 3 * n, vel, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, h->st));
            dvel = stg + 3 * n;
        }
    }
    const Parts P = parts_of(h);
    jt_launch_split_signed(dpos, dvel, h->sign_caller, (int64_t)n, h->rank_buf, P.pos[0], P.vel[0],
                           P.id[0], h->gmap[0], P.pos[1], P.vel[1], P.id[1], h->gmap[1], h->st);
    JT_CU(cudaStreamSynchronize(h->st));
    JT_CU(cudaGetLastError());
    h->signed_layout = true;
    h->have_state = true;
    return JT_OK;
}

namespace {

// One force evaluation at the current positions (no kick), any mode.
int force_only(jt_handle* h, int part)
{
    if (h->batch) {
        jtb_reset_timings(h->batch);
        return jtb_force_pass(h->batch, &h->box_id, 1, part, 0.0f, nullptr);
    }
    return compute_forces_rc(h, 0.0f, 0.0f, part);
}

// Wait for the call's work, read the device error word, collect timings.
int finish_call(jt_handle* h, int r, cudaEvent_t t0, cudaEvent_t t1)
{
    int e;
    if (h->batch) {
        e = jtb_finish(h->batch);
        if (e == JT_OK) jt_batch_get_timings(h->batch, &h->tm);
        for (int i = 0; i < 4; i++) h->phase[i] = jtb_phase(h->batch, i);
    } else {
        e = check_device_error(h);
        if (e == JT_OK) {
            accumulate_timings(h);
            fetch_inter(h);
        }
    }
    if (r == JT_OK) r = e;
    if (r == JT_OK && t0 && t1) h->tm.total_ms = elapsed(t0, t1);
    return r;
}

}  // namespace

int jt_accel(jt_handle* h, float* acc_p, float* acc_m, int mem)
{
    return jt_accel_part(h, JT_PART_ALL, acc_p, acc_m, mem);
}

int jt_accel_part(jt_handle* h, int part, float* acc_p, float* acc_m, int mem)
{
    if (!h || (mem != JT_MEM_HOST && mem != JT_MEM_DEVICE)) return JT_EINVAL;
    if (part < 1 || part > 3) return JT_EINVAL;
    if (!h->have_state) return JT_ESTATE;
    if (h->signed_layout) return JT_EINVAL;  // state loaded with the signed layout: jt_accel_signed
    h->tm = jt_timings{};
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaEventRecord(t0, h->st);
    int r = force_only(h, part);
    cudaEventRecord(t1, h->st);
    if (r == JT_OK) {
        const Parts P = parts_of(h);
        r = write_out(h, P.acc[0], P.id[0], nullptr, h->n[0], acc_p, mem);
        if (r == JT_OK) {
            // the host path reuses the staging buffer: finish the first copy
            if (mem == JT_MEM_HOST) cudaStreamSynchronize(h->st);
            r = write_out(h, P.acc[1], P.id[1], nullptr, h->n[1], acc_m, mem);
        }
    }
    r = finish_call(h, r, t0, t1);
    if (part != JT_PART_ALL) {
        h->acc_valid = false;
        if (h->batch) jtb_box(h->batch, h->box_id)->acc_valid = false;
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    return r;
}

int jt_accel_signed(jt_handle* h, float* acc, int mem)
{
    if (!h || !acc || (mem != JT_MEM_HOST && mem != JT_MEM_DEVICE)) return JT_EINVAL;
    if (!h->have_state) return JT_ESTATE;
    h->tm = jt_timings{};
    int r = force_only(h, JT_PART_ALL);
    if (r == JT_OK) {
        const Parts P = parts_of(h);
        int64_t na = h->n[0] + h->n[1];
        float* target = mem == JT_MEM_DEVICE ? acc : (float*)h->stage;
        for (int s = 0; s < 2; s++) jt_launch_aos_out(P.acc[s], P.id[s], h->gmap[s], h->n[s], target, h->st);
        if (mem == JT_MEM_HOST)
            cudaMemcpyAsync(acc, h->stage, sizeof(float) * 3 * na, cudaMemcpyDeviceToHost, h->st);
    }
    return finish_call(h, r, nullptr, nullptr);
}

int jt_step(jt_handle* h, double dt, double hubble, double dtau_per_dt, int nsteps)
{
    if (!h || nsteps < 0 || !std::isfinite(dt) || !std::isfinite(hubble) || !std::isfinite(dtau_per_dt))
        return JT_EINVAL;
    if (!h->have_state) return JT_ESTATE;
    if (nsteps == 0) return JT_OK;
    h->tm = jt_timings{};
    const jt_config& c = h->cfg;
    if (h->batch && c.integrator == JT_KDK) {
        jt_step_args a;
        a.dt = dt;
        a.hubble = hubble;
        a.dtau_per_dt = dtau_per_dt;
        int r = jt_batch_step(h->batch, &h->box_id, 1, &a, nsteps);
        jt_batch_get_timings(h->batch, &h->tm);
        for (int i = 0; i < 4; i++) h->phase[i] = jtb_phase(h->batch, i);
        return r;
    }
    // FP64 step factors, applied in FP32
    const double drag_d = hubble * dtau_per_dt;
    const float drag = (float)drag_d;
    const float L = (float)c.box_L, halfL = (float)(c.box_L / 2.0);
    const float half = (float)(0.5 * dt), full = (float)dt;
    cudaEvent_t t0, t1, k0, k1;
    cudaEventCreate(&t0); cudaEventCreate(&t1); cudaEventCreate(&k0); cudaEventCreate(&k1);
    cudaEventRecord(t0, h->st);
    int r = JT_OK;
    double kd_ms = 0.0;
    jt_timings acc_tm = {};
    auto add_pass = [&](void) {
        // stage times of one force pass (batch timings are per pass)
        if (!h->batch) return;
        jt_timings t;
        jt_batch_get_timings(h->batch, &t);
        acc_tm.sort_ms += t.sort_ms; acc_tm.tree_ms += t.tree_ms; acc_tm.deposit_ms += t.deposit_ms;
        acc_tm.fft_ms += t.fft_ms; acc_tm.kspace_ms += t.kspace_ms; acc_tm.walk_ms += t.walk_ms;
        acc_tm.interactions += t.interactions; acc_tm.launches += t.launches;
        acc_tm.pair_interactions += t.pair_interactions; acc_tm.node_interactions += t.node_interactions;
        acc_tm.candidates += t.candidates;
        acc_tm.cellwalk_ms += t.cellwalk_ms;
        acc_tm.interp_ms += t.interp_ms;
    };
    if (c.integrator == JT_KDK) {
        // RCOMPAT kick-drift-kick (the accurate handle went through the batch)
        if (!h->acc_valid) {
            r = compute_forces_rc(h, 0.0f, 0.0f);
            if (r == JT_OK) r = finish_call(h, r, nullptr, nullptr);
        }
        for (int k = 0; k < nsteps && r == JT_OK; k++) {
            cudaEventRecord(k0, h->st);
            for (int s = 0; s < 2; s++) {
                jt_launch_kick(h->vel[s], h->acc[s], h->n[s], half, drag, h->st);
                jt_launch_drift(h->pos[s], h->vel[s], h->n[s], full, L, halfL, h->st);
            }
            cudaEventRecord(k1, h->st);
            r = compute_forces_rc(h, half, drag);
            if (r != JT_OK) break;
            r = finish_call(h, r, nullptr, nullptr);
            kd_ms += elapsed(k0, k1);
        }
    } else {
        // the reference's drift(dt/2) force kick(dt) drift(dt/2)
        for (int k = 0; k < nsteps && r == JT_OK; k++) {
            cudaEventRecord(k0, h->st);
            Parts P = parts_of(h);
            for (int s = 0; s < 2; s++) jt_launch_drift(P.pos[s], P.vel[s], h->n[s], half, L, halfL, h->st);
            cudaEventRecord(k1, h->st);
            r = force_only(h, JT_PART_ALL);
            if (r != JT_OK) break;
            P = parts_of(h);
            for (int s = 0; s < 2; s++) {
                jt_launch_kick(P.vel[s], P.acc[s], h->n[s], full, drag, h->st);
                jt_launch_drift(P.pos[s], P.vel[s], h->n[s], half, L, halfL, h->st);
            }
            r = finish_call(h, r, nullptr, nullptr);
            add_pass();
            kd_ms += elapsed(k0, k1);
            h->acc_valid = false;  // acc belongs to the half-drifted positions
            if (h->batch) jtb_box(h->batch, h->box_id)->acc_valid = false;
        }
    }
    cudaEventRecord(t1, h->st);
    if (cudaStreamSynchronize(h->st) != cudaSuccess && r == JT_OK) r = JT_ECUDA;
    if (h->batch) h->tm = acc_tm;
    if (r == JT_OK) {
        h->tm.total_ms = elapsed(t0, t1);
        h->tm.kick_drift_ms = kd_ms;
    }
    cudaEventDestroy(t0); cudaEventDestroy(t1); cudaEventDestroy(k0); cudaEventDestroy(k1);
    return r;
}

int jt_step_host(jt_handle* h, float* pos_p, float* vel_p, float* acc_p, float* pos_m, float* vel_m,
                 float* acc_m, double dt, double hubble, double dtau_per_dt)
{
    if (!h || !std::isfinite(dt) || !std::isfinite(hubble) || !std::isfinite(dtau_per_dt)) return JT_EINVAL;
    if (!h->have_state) return JT_ESTATE;
    if (h->signed_layout) return JT_EINVAL;
    const bool kdk = h->cfg.integrator == JT_KDK;
    float* pos[2] = {pos_p, pos_m};
    float* vel[2] = {vel_p, vel_m};
    float* acc[2] = {acc_p, acc_m};
    for (int s = 0; s < 2; s++)
        if (h->n[s] > 0 && (!pos[s] || !vel[s] || (kdk && !acc[s]))) return JT_EINVAL;
    if (h->batch && kdk) {
        h->tm = jt_timings{};
        const int r = jtb_step_host(h->batch, h->box_id, pos, vel, acc, (float)dt, (float)(hubble * dtau_per_dt));
        jt_batch_get_timings(h->batch, &h->tm);
        for (int i = 0; i < 4; i++) h->phase[i] = jtb_phase(h->batch, i);
        return r;
    }
    // compatibility mode and the reference's DKD: the same round trip
    // through the separate calls (no overlap)
    JT_TRY(jt_set_state(h, pos_p, vel_p, (size_t)h->n[0], pos_m, vel_m, (size_t)h->n[1], JT_MEM_HOST));
    if (kdk) JT_TRY(jt_set_accel(h, acc_p, acc_m, JT_MEM_HOST));
    JT_TRY(jt_step(h, dt, hubble, dtau_per_dt, 1));
    const jt_timings tm = h->tm;
    JT_TRY(jt_get_state(h, pos_p, vel_p, pos_m, vel_m, JT_MEM_HOST));
    if (kdk) JT_TRY(jt_get_accel(h, acc_p, acc_m, JT_MEM_HOST));
    h->tm = tm;
    return JT_OK;
}

int jt_set_accel(jt_handle* h, const float* acc_p, const float* acc_m, int mem)
{
    if (!h || (mem != JT_MEM_HOST && mem != JT_MEM_DEVICE)) return JT_EINVAL;
    if (!h->have_state) return JT_ESTATE;
    if (h->signed_layout) return JT_EINVAL;
    const float* src[2] = {acc_p, acc_m};
    for (int s = 0; s < 2; s++)
        if (h->n[s] > 0 && !src[s]) return JT_EINVAL;
    const Parts P = parts_of(h);
    for (int s = 0; s < 2; s++) {
        const int64_t n = h->n[s];
        if (n == 0) continue;
        void* d = nullptr;
        JT_TRY(copy_in(h, src[s], sizeof(float) * 3 * (size_t)n, mem, &d));
        k_aos_gather<<<(unsigned)((n + 255) / 256), 256, 0, h->st>>>((const float*)d, P.id[s], n, P.acc[s]);
        JT_CU(cudaGetLastError());
        JT_CU(cudaStreamSynchronize(h->st));   // the staging buffer is reused
    }
    h->tm.launches += (h->n[0] > 0) + (h->n[1] > 0);
    h->acc_valid = true;
    if (h->batch) jtb_box(h->batch, h->box_id)->acc_valid = true;
    return JT_OK;
}

int jt_get_accel(jt_handle* h, float* acc_p, float* acc_m, int mem)
{
    if (!h || (mem != JT_MEM_HOST && mem != JT_MEM_DEVICE)) return JT_EINVAL;
    if (!h->have_state) return JT_ESTATE;
    if (h->signed_layout) return JT_EINVAL;
    const bool valid = h->batch ? jtb_box(h->batch, h->box_id)->acc_valid : h->acc_valid;
    if (!valid) return JT_ESTATE;
    const Parts P = parts_of(h);
    JT_TRY(write_out(h, P.acc[0], P.id[0], nullptr, h->n[0], acc_p, mem));
    if (mem == JT_MEM_HOST) JT_CU(cudaStreamSynchronize(h->st));
    JT_TRY(write_out(h, P.acc[1], P.id[1], nullptr, h->n[1], acc_m, mem));
    JT_CU(cudaStreamSynchronize(h->st));
    return JT_OK;
}

int jt_set_counters(jt_handle* h, int on)
{
    if (!h) return JT_EINVAL;
    return h->batch ? jt_batch_set_counters(h->batch, on) : JT_OK;
}

int jt_set_screening(jt_handle* h, double lambda_0, double z)
{
    if (!h || !(lambda_0 >= 0.0) || !(z > -1.0) || !std::isfinite(lambda_0) || !std::isfinite(z))
        return JT_EINVAL;
    if (h->batch && h->box_id >= 0) JT_TRY(jt_batch_set_screening(h->batch, h->box_id, lambda_0, z));
    if (h->lambda_0 != lambda_0 || h->z != z) h->acc_valid = false;
    h->lambda_0 = lambda_0;
    h->z = z;
    return JT_OK;
}

int jt_get_state(jt_handle* h, float* pos_p, float* vel_p, float* pos_m, float* vel_m, int mem)
{
    if (!h || (mem != JT_MEM_HOST && mem != JT_MEM_DEVICE)) return JT_EINVAL;
    if (!h->have_state) return JT_ESTATE;
    const Parts P = parts_of(h);
    float* outs[2][2] = {{pos_p, vel_p}, {pos_m, vel_m}};
    for (int s = 0; s < 2; s++) {
        for (int q = 0; q < 2; q++) {
            JT_TRY(write_out(h, q == 0 ? P.pos[s] : P.vel[s], P.id[s], nullptr, h->n[s], outs[s][q], mem));
            JT_CU(cudaStreamSynchronize(h->st));
        }
    }
    return JT_OK;
}

int jt_get_state_signed(jt_handle* h, float* pos, float* vel, int mem)
{
    if (!h || (mem != JT_MEM_HOST && mem != JT_MEM_DEVICE)) return JT_EINVAL;
    if (!h->have_state) return JT_ESTATE;
    const Parts P = parts_of(h);
    int64_t na = h->n[0] + h->n[1];
    float* outs[2] = {pos, vel};
    for (int q = 0; q < 2; q++) {
        if (!outs[q]) continue;
        float* target = mem == JT_MEM_DEVICE ? outs[q] : (float*)h->stage;
        for (int s = 0; s < 2; s++)
            jt_launch_aos_out(q == 0 ? P.pos[s] : P.vel[s], P.id[s], h->gmap[s], h->n[s], target, h->st);
        if (mem == JT_MEM_HOST)
            JT_CU(cudaMemcpyAsync(outs[q], h->stage, sizeof(float) * 3 * na, cudaMemcpyDeviceToHost, h->st));
        JT_CU(cudaStreamSynchronize(h->st));
    }
    return JT_OK;
}

int jt_debug_tree(jt_handle* h, int species, uint32_t* morton, int32_t* perm, int32_t* left,
                  int32_t* right, int32_t* parent)
{
    if (!h || species < 0 || species > 1) return JT_EINVAL;
    if (!h->have_state) return JT_ESTATE;
    int64_t n = h->n[species];
    if (n == 0) return JT_OK;
    if (!h->dbg_ready) JT_TRY(alloc_trees(h, h->n[0], h->n[1]));
    const Parts P = parts_of(h);
    jt_tree_dev& t = h->tree[species];
    float box_half = (float)(h->cfg.box_L / 2.0);
    // reference keys at the current positions, without moving the state
    jt_launch_morton(P.pos[species], P.id[species], n, box_half, nullptr, h->key64, h->ws.vals, h->st);
    int shifts[8], np = 0;
    for (int b = 0; b < id_bits(n); b += 8) shifts[np++] = b;
    for (int b = 32; b < 62; b += 8) shifts[np++] = b;
    JT_TRY(jt_radix_sort_u64(h->key64, h->ws.vals, n, shifts, np, &h->ws, h->d_err, h->st));
    jt_launch_split_keys(h->key64, n, t.m30, t.tie, h->st);
    jt_tree_dev tk = t;
    tk.n = n;
    jt_launch_karras(tk, h->st);
    JT_TRY(check_device_error(h));
    int64_t nn = 2 * n - 1;
    std::vector<int2> ch(nn);
    if (morton) JT_CU(cudaMemcpy(morton, t.m30, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost));
    if (perm) JT_CU(cudaMemcpy(perm, t.tie, sizeof(int32_t) * n, cudaMemcpyDeviceToHost));
    JT_CU(cudaMemcpy(ch.data(), t.child, sizeof(int2) * nn, cudaMemcpyDeviceToHost));
    if (parent) JT_CU(cudaMemcpy(parent, t.parent, sizeof(int32_t) * nn, cudaMemcpyDeviceToHost));
    for (int64_t i = 0; i < nn; i++) {
        if (left) left[i] = ch[i].x;
        if (right) right[i] = ch[i].y;
    }
    // RCOMPAT: the tree arrays no longer describe the state order; the next
    // force evaluation rebuilds them
    h->acc_valid = false;
    return JT_OK;
}

}  // extern "C"

namespace {
__global__ void k_scale_vel4(float4* __restrict__ v, int64_t n, float a)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float4 q = v[i];
    q.x *= a;
    q.y *= a;
    q.z *= a;
    v[i] = q;
}
}  // namespace

// Multiply every velocity by a, in place (internal order: the product does
// not depend on it).
int jth_scale_velocities(jt_handle* h, float a)
{
    if (!h || !h->have_state) return JT_ESTATE;
    Parts P = parts_of(h);
    for (int s = 0; s < 2; s++)
        if (h->n[s] > 0)
            k_scale_vel4<<<(unsigned)((h->n[s] + 255) / 256), 256, 0, h->st>>>(P.vel[s], h->n[s], a);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(h->st) != cudaSuccess) return JT_ECUDA;
    h->tm.launches += (h->n[0] > 0) + (h->n[1] > 0);
    return JT_OK;
}

int jth_info(jt_handle* h, jt_config* cfg, float* m_plus, float* m_minus, int8_t* signs)
{
    if (!h) return JT_EINVAL;
    if (!h->have_state) return JT_ESTATE;
    if (cfg) *cfg = h->cfg;
    if (m_plus) *m_plus = h->mass[0];
    if (m_minus) *m_minus = h->mass[1];
    if (signs && cudaMemcpy(signs, h->sign_caller, (size_t)(h->n[0] + h->n[1]), cudaMemcpyDeviceToHost) != cudaSuccess)
        return JT_ECUDA;
    return JT_OK;
}

extern "C" {

int jt_diagnostics(jt_handle* h, int n_cells, jt_diag* out)
{
    if (!h || !out) return JT_EINVAL;
    if (!h->have_state) return JT_ESTATE;
    const Parts P = parts_of(h);
    const float4* pos[2] = {P.pos[0], P.pos[1]};
    const float4* vel[2] = {P.vel[0], P.vel[1]};
    return jt_diag_state(pos, vel, h->n, h->mass, h->cfg.box_L, n_cells, h->st, out);
}

int jt_walk_counters(jt_handle* h, int64_t* out4)
{
    if (!h || !out4) return JT_EINVAL;
    for (int i = 0; i < 4; i++) out4[i] = h->phase[i];
    return JT_OK;
}

int jt_get_timings(jt_handle* h, jt_timings* t)
{
    if (!h || !t) return JT_EINVAL;
    *t = h->tm;
    return JT_OK;
}

int jt_counts(jt_handle* h, size_t* n_p, size_t* n_m)
{
    if (!h) return JT_EINVAL;
    if (n_p) *n_p = (size_t)h->n[0];
    if (n_m) *n_m = (size_t)h->n[1];
    return JT_OK;
}

}  // extern "C"
