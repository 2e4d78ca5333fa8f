// Batched engine: many independent boxes advanced with ONE launch per stage.
//
// The reference runs parameter scans one box at a time, one process per
// configuration (optim/run_tour.py:40-48, scripts/run_scan_mu.sh), each box
// paying its own ~40 launches and host synchronisations per step
// (src/nbody_gpu_twopass.rs:4486-4649).  Here a jt_batch holds any number of
// boxes (uneven particle counts, box sizes, PM grids, mu); a step over a
// chosen subset of them runs every stage as one launch over the flattened
// work of all chosen boxes (segments = box x species, jt_internal.cuh), with
// cuFFT plans bucketed by grid size (batched R2C and C2R per
// distinct M).  Only particle state persists per box; trees, sort workspaces
// and PM grids are per-pass scratch in grow-only pools, so boxes can join and
// leave between steps (the serving loop admits and evicts jobs this way).
//
// Per force pass (stream order, no host synchronisation inside):
//   memset sort status -> morton, hist, scan, 4 onesweep passes, reorder
//   (8 launches over all segments) -> karras, moments (2) -> memset rho per
//   grid bucket -> tile ranges, tiled deposit (2) -> R2C per bucket ->
//   k-space (1) -> C2R per bucket -> walk with fused closing kick (1).
#include "jt_batch.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

namespace {

#define JT_TRY(x)                   \
    do {                            \
        int _r = (x);               \
        if (_r != JT_OK) return _r; \
    } while (0)
#define JT_CU(x)                                 \
    do {                                         \
        if ((x) != cudaSuccess) return JT_ECUDA; \
    } while (0)
#define JT_FFT(x)                                  \
    do {                                           \
        if ((x) != CUFFT_SUCCESS) return JT_ECUDA; \
    } while (0)

// Device memory of a batch comes from its own stream-ordered pool
// (cudaMallocFromPoolAsync / cudaFreeAsync on the batch's stream), which
// keeps freed blocks for reuse: admitting and evicting boxes, growing pools
// and trimming them never synchronise the device.  Every entry point that
// may allocate or free sets the batch as the calling thread's allocation
// context (AllocScope); a batch is used by one host thread at a time.
struct AllocCtx {
    cudaMemPool_t pool = nullptr;
    cudaStream_t st = nullptr;
};
thread_local const AllocCtx* t_alloc = nullptr;

struct AllocScope {
    const AllocCtx* prev;
    explicit AllocScope(const AllocCtx* c) : prev(t_alloc) { t_alloc = c; }
    ~AllocScope() { t_alloc = prev; }
};

template <class T>
int dalloc(T** p, size_t count)
{
    *p = nullptr;
    if (!t_alloc) return JT_EINVAL;
    if (count == 0) count = 1;
    if (cudaMallocFromPoolAsync((void**)p, sizeof(T) * count, t_alloc->pool, t_alloc->st) == cudaSuccess)
        return JT_OK;
    *p = nullptr;
    cudaGetLastError();   // an allocation failure is not sticky: keep it out of later checks
    return JT_ENOMEM;
}
template <class T>
void dfree(T*& p)
{
    if (p && t_alloc) cudaFreeAsync((void*)p, t_alloc->st);
    p = nullptr;
}

// grow-only device array (1/16 headroom on growth)
template <class T>
struct Pool {
    T* p = nullptr;
    size_t cap = 0;
    int ensure(size_t n, bool* grew)
    {
        if (n <= cap) return JT_OK;
        size_t want = std::max(n, cap + cap / 16);
        dfree(p);
        cap = 0;
        JT_TRY(dalloc(&p, want));
        cap = want;
        *grew = true;
        return JT_OK;
    }
    size_t bytes() const { return cap * sizeof(T); }
    void release()
    {
        dfree(p);
        cap = 0;
    }
};

int box_order(const jt_config& c) { return c.pm_order == 0 ? 4 : c.pm_order; }
int box_ngrid(const jt_config& c) { return c.pm_interlace == 2 ? 1 : 2; }

// One allocation of a bucket's grid arrays: `slots` boxes, each with its
// ngrid density grids and spectra and 3 ngrid force spectra and grids.
struct BucketChunk {
    int slots = 0;
    float* rho = nullptr;
    float2* rho_k = nullptr;
    float2* force_k = nullptr;
    float* force = nullptr;
    int4* ranges = nullptr;
    void free_arrays()
    {
        dfree(rho); dfree(rho_k); dfree(force_k); dfree(force); dfree(ranges);
        slots = 0;
    }
};

struct Bucket {                 // PM scratch of the boxes with grid M in a pass
    int M = 0;
    int cap = 0;                // boxes the chunks hold
    // z transforms fused with the k-space step (jt_zfft.cu): cuFFT's plans
    // are 2D, one transform per (x, y) plane; fixed when the bucket is made
    bool fused = false;
    bool decided = false;
    // The grid arrays, in chunks: a pass with more boxes of this grid than
    // the chunks hold adds one chunk for the missing slots and leaves the
    // others in place.  (Freeing and allocating the whole bucket at the new
    // count made the pool map several GB per 512^3 box while the step
    // waited: up to ~1 s with the device idle when served jobs arrive a few
    // at a time.)  Slot q of a pass is in the first chunk whose running
    // count exceeds q; cuFFT's batches never cross a chunk.
    std::vector<BucketChunk> chunks;
    // batched plans by transform count: r2c[b], c2r[b] transform b grids
    // per execution (at most fft_chunk(M) each, see below)
    std::map<int, cufftHandle> r2c, c2r;
    void free_arrays()
    {
        for (auto& c : chunks) c.free_arrays();
        chunks.clear();
        cap = 0;
    }
    // the chunk holding slot q and q's index in it
    const BucketChunk& locate(int q, int* i) const
    {
        size_t c = 0;
        while (c + 1 < chunks.size() && q >= chunks[c].slots) {
            q -= chunks[c].slots;
            c++;
        }
        *i = q;
        return chunks[c];
    }
    void release()
    {
        free_arrays();
        for (auto& kv : r2c) cufftDestroy(kv.second);
        for (auto& kv : c2r) cufftDestroy(kv.second);
        r2c.clear();
        c2r.clear();
    }
};

size_t grid_bytes(int64_t M, int ngrid)
{
    int64_t G = M * M * M, Gc = M * M * (M / 2 + 1);
    int T = jt_pm_tile_edge((int)M);
    int64_t nt = (M / T) * (M / T) * (M / T);
    return (size_t)(ngrid * (G * 4 + Gc * 8) + 3 * ngrid * (Gc * 8 + G * 4) + nt * 16);
}

// The tables of one pass, packed into one host buffer and uploaded once.
// the near-field cell walk (on unless JT_WALK_CELLS=0, which keeps the tree
// walk for every particle)
bool cells_enabled()
{
    const char* e = std::getenv("JT_WALK_CELLS");
    return !(e && e[0] == '0');
}

struct Plan {
    std::vector<int> ids;                 // boxes of this pass
    std::vector<jt_seg_dev> pre, post;    // segments before / after the reorder
    std::vector<jt_box_dev> bx;
    std::vector<int64_t> pprefix, iprefix, tprefix, gprefix, ptprefix, kprefix, cprefix, zprefix;
    int64_t npart = 0, ninternal = 0, nsorttiles = 0, ngroups = 0, npmtiles = 0, nmodes = 0, ncells = 0;
    int64_t nztiles = 0;                  // CTAs of the fused z-transform kernel
    int zsizes = 0;                       // its grid sizes in the pass: bit 0 512^3, bit 1 256^3
    bool cells = false;                   // the near-field cell walk runs (jt_b_cells)
    bool screened = false;                // some box is screened (second source, Yukawa tables)
    std::map<int, std::vector<int>> by_M; // M -> boxes (positions in ids)
    std::map<int, int> nslots;            // M -> bucket slots (a screened box takes two: D, then S)
    int maxT = 1, minT = 1 << 30;
    size_t table_bytes = 0;
    const jt_seg_dev* d_pre = nullptr;
    const jt_seg_dev* d_post = nullptr;
    const jt_box_dev* d_bx = nullptr;
    const int64_t *d_pp = nullptr, *d_ip = nullptr, *d_tp = nullptr, *d_gp = nullptr, *d_ptp = nullptr,
                  *d_kp = nullptr, *d_cp = nullptr, *d_zp = nullptr;
};

float elapsed(cudaEvent_t a, cudaEvent_t b)
{
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) return 0.f;
    return ms;
}

}  // namespace

struct jt_batch {
    int device = 0;
    jt_ckpt* ckpt = nullptr;            // asynchronous checkpoint (jt_ckpt.cu)
    cudaStream_t st = nullptr;
    AllocCtx actx;                      // its memory pool and stream
    Pool<float> stage;                  // host <-> device staging of AoS arrays
    // jtb_step_host: the uploaded and outgoing state (per species pos | vel |
    // acc, AoS float3) and the side stream that copies positions back
    Pool<float> io;
    cudaStream_t io_side = nullptr;
    cudaEvent_t io_ev = nullptr;
    std::vector<jt_box_state*> boxes;
    int order = 0, ngrid = 0, k_min = -1;   // shared by every box of the batch
    Pool<int2> child, range;
    Pool<int> parent, flag;
    // near-field cell list (jt_b_cells)
    Pool<int> ccount, cstart, cbsum, ccell, csegflag;
    Pool<unsigned> cslot;
    Pool<float4> cpos;
    Pool<float4> pmacc;                 // PM accelerations of the pass, per interlaced grid
    Pool<int2> cid;
    Pool<unsigned char> tflag;
    Pool<float4> com, bmin, bmax, quad0;
    Pool<float2> quad1;
    Pool<uint32_t> m30, vals, vals_alt, keys_alt, hist, status, tickets;
    Pool<unsigned char> desc;           // device copy of the pass's tables
    unsigned char* hdesc = nullptr;     // pinned host staging of the tables
    size_t hdesc_cap = 0;
    cudaEvent_t desc_done = nullptr;    // the last upload from hdesc finished
    std::map<int, Bucket> buckets;
    unsigned* d_err = nullptr;
    unsigned long long* d_stats = nullptr;
    cudaEvent_t ev[11] = {};            // 8, 9: around the cell walk kernel; 6-10: interpolation
    bool counters = false;              // the cell walk counts its pairs (jt_batch_set_counters)
    bool cell_tune = true;              // tune_cells may run (jtb_set_cell_tune)
    bool pending = false;               // a pass's events await jtb_finish
    jt_timings tm = {};
    int64_t phase[4] = {0, 0, 0, 0};
    Plan plan;
    // CUDA graphs of one step (opt-in, jt_batch_set_graphs)
    uint64_t gen = 0;                   // bumps when an address a captured plan holds may change
    bool use_graphs = false;
    struct {
        std::vector<int> ids;
        uint64_t gen = ~0ull;
        Plan plan;                      // its tables live in gdesc
        cudaGraphExec_t exec[2] = {nullptr, nullptr};
        const float4* pre0 = nullptr;   // first segment's pos at parity 0
        int box0 = -1, sp0 = 0;
        int64_t launches = 0;           // kernels per replay
    } gc;
    Pool<unsigned char> gdesc;
    // one cuFFT work area shared by every plan (they run in stream order)
    Pool<unsigned char> fftws;
    size_t fft_need = 0;
    bool fft_dirty = false;
};

namespace {

// Per-axis k tables of a box (index n = 0..M-1), computed on the device so
// that adding a box needs no host-to-device copy from pageable memory (which
// would wait for the batch's stream):
//   ta = {k, gradient k (0 at Nyquist), exp(-k^2 r_s^2) / sinc^(2 order), |n|}
//   tb = {cos(k h / 2), sin(k h / 2), 0, 0} (interlacing phase)
__global__ void k_box_tabs(float4* __restrict__ tabs, int M, double L, double rs, int order)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= M) return;
    const int ni = n <= M / 2 ? n : n - M;
    const double dk = 2.0 * M_PI / L, hh = L / M;
    const double k = dk * ni;
    const double u = M_PI * ni / M;
    const double sinc = ni == 0 ? 1.0 : sin(u) / u;
    double w = 1.0;
    for (int i = 0; i < 2 * order; i++) w *= sinc;
    const double f = exp(-k * k * rs * rs) / w;
    tabs[n] = make_float4((float)k, n == M / 2 ? 0.0f : (float)k, (float)f, (float)(ni < 0 ? -ni : ni));
    tabs[M + n] = make_float4((float)cos(0.5 * k * hh), (float)sin(0.5 * k * hh), 0.0f, 0.0f);
}

int box_alloc(jt_box_state* b)
{
    size_t bytes = 0;
    for (int s = 0; s < 2; s++) {
        int64_t n = b->n[s];
        JT_TRY(dalloc(&b->pos[s], n)); JT_TRY(dalloc(&b->vel[s], n)); JT_TRY(dalloc(&b->acc[s], n));
        JT_TRY(dalloc(&b->pos_b[s], n)); JT_TRY(dalloc(&b->vel_b[s], n));
        JT_TRY(dalloc(&b->id[s], n)); JT_TRY(dalloc(&b->id_b[s], n));
        bytes += (size_t)n * (5 * sizeof(float4) + 2 * sizeof(int));
    }
    const int M = b->M;
    JT_TRY(dalloc(&b->tabs, 2 * (size_t)M));
    const jt_config& c = b->cfg;
    k_box_tabs<<<(M + 127) / 128, 128, 0, t_alloc->st>>>(b->tabs, M, c.box_L, c.r_s, b->order);
    JT_CU(cudaGetLastError());
    b->bytes = bytes + sizeof(float4) * 2 * (size_t)M;
    return JT_OK;
}

void box_release(jt_box_state* b)
{
    for (int s = 0; s < 2; s++) {
        dfree(b->pos[s]); dfree(b->vel[s]); dfree(b->acc[s]); dfree(b->pos_b[s]); dfree(b->vel_b[s]);
        dfree(b->id[s]); dfree(b->id_b[s]);
    }
    dfree(b->tabs);
    dfree(b->ytab);
    b->kappa = 0.0;
}

int tile_shift_of(int M)
{
    int T = jt_pm_tile_edge(M);
    int W = 1024 / M * T;  // tile edge in Morton cells (power of two)
    int lw = 0;
    while ((1 << lw) < W) lw++;
    return 3 * lw;
}

// Grids per cuFFT execution: at most 2^27 real elements (one 512^3 grid,
// eight 256^3, ...), which keeps every plan inside cuFFT's 32-bit sizes and
// bounds its work area; a bucket's transforms run as consecutive chunks.
int fft_chunk(int M)
{
    const int64_t G = (int64_t)M * M * M;
    const int64_t c = ((int64_t)1 << 27) / G;
    return c < 1 ? 1 : (int)c;
}

// fused: the grids' (x, y) planes as 2D transforms, M per grid
int make_plan(jt_batch* B, std::map<int, cufftHandle>& pl, int M, int batch, bool r2c, bool fused)
{
    if (batch <= 0 || pl.count(batch)) return JT_OK;
    const int64_t G = (int64_t)M * M * M, Gc = (int64_t)M * M * (M / 2 + 1);
    int dims[3] = {M, M, M};
    const int rank = fused ? 2 : 3;
    const int64_t rd = fused ? (int64_t)M * M : G, cd = fused ? (int64_t)M * (M / 2 + 1) : Gc;
    const int n = fused ? batch * M : batch;
    cufftHandle h;
    if (cufftCreate(&h) != CUFFT_SUCCESS) return JT_ECUDA;
    // the work area is the batch's shared one (set once all plans exist)
    cufftSetAutoAllocation(h, 0);
    size_t ws = 0;
    cufftResult e = r2c ? cufftMakePlanMany(h, rank, dims, nullptr, 1, (int)rd, nullptr, 1, (int)cd, CUFFT_R2C,
                                            n, &ws)
                        : cufftMakePlanMany(h, rank, dims, nullptr, 1, (int)cd, nullptr, 1, (int)rd, CUFFT_C2R,
                                            n, &ws);
    if (e != CUFFT_SUCCESS) {
        cufftDestroy(h);
        cudaGetLastError();
        return e == CUFFT_ALLOC_FAILED ? JT_ENOMEM : JT_ECUDA;
    }
    cufftSetStream(h, B->st);
    B->fft_need = std::max(B->fft_need, ws);
    B->fft_dirty = true;
    pl[batch] = h;
    return JT_OK;
}

// 512^3 grids take the fused z path unless JT_ZFFT=0 (read when a bucket is
// made: the old path stays reachable for comparisons)
bool zfft_for(int M)
{
    if (jt_zfft_tiles(M) == 0) return false;
    const char* e = std::getenv("JT_ZFFT");
    return !(e && e[0] == '0');
}

int bucket_ensure(jt_batch* B, Bucket& k, int M, int count)
{
    k.M = M;
    if (!k.decided) {
        k.fused = zfft_for(M);
        k.decided = true;
    }
    const int ngrid = B->ngrid;
    const int64_t G = (int64_t)M * M * M, Gc = (int64_t)M * M * (M / 2 + 1);
    if (count > k.cap) {
        B->gen++;
        int T = jt_pm_tile_edge(M);
        int64_t nt = (int64_t)(M / T) * (M / T) * (M / T);
        const int add = count - k.cap;
        BucketChunk c;
        c.slots = add;
        int r = dalloc(&c.rho, (size_t)add * ngrid * G);
        if (r == JT_OK) r = dalloc(&c.rho_k, (size_t)add * ngrid * Gc);
        if (r == JT_OK) r = dalloc(&c.force_k, (size_t)add * 3 * ngrid * Gc);
        if (r == JT_OK) r = dalloc(&c.force, (size_t)add * 3 * ngrid * G);
        if (r == JT_OK) r = dalloc(&c.ranges, (size_t)add * nt);
        if (r != JT_OK) {
            c.free_arrays();
            return r;
        }
        k.chunks.push_back(c);
        k.cap = count;
    }
    // plans for every power-of-two batch the executions of this count use:
    // the executions run chunk by chunk (exec_r2c, exec_c2r), each chunk's
    // share of the count as full batches of fft_chunk(M) grids (a power of
    // two) and the remainder's binary decomposition, so a bucket holds at
    // most log2(fft_chunk) + 1 plans per direction whatever counts later
    // passes bring (creating a plan inside a pass costs more than the
    // transforms; the server makes them all at registration)
    const int ch = fft_chunk(M);
    int left = count;
    for (const BucketChunk& C : k.chunks) {
        if (left <= 0) break;
        const int u = std::min(left, C.slots);
        left -= u;
        for (int dir = 0; dir < 2; dir++) {
            const int n = (dir == 0 ? ngrid : 3 * ngrid) * u;
            auto& pl = dir == 0 ? k.r2c : k.c2r;
            if (n >= ch) JT_TRY(make_plan(B, pl, M, ch, dir == 0, k.fused));
            for (int b = 1; b < ch; b <<= 1)
                if ((n % ch) & b) JT_TRY(make_plan(B, pl, M, b, dir == 0, k.fused));
        }
    }
    return JT_OK;
}

// largest batch of one execution for n transforms left: a full chunk, else
// the highest power of two in n
int fft_batch(int n, int ch)
{
    if (n >= ch) return ch;
    int b = 1;
    while (b * 2 <= n) b <<= 1;
    return b;
}

// Run n transforms of a bucket in chunks of at most fft_chunk(M).
// the density grids of the pass's first `slots` slots, chunk by chunk
int exec_r2c(Bucket& K, int slots, int ngrid)
{
    const int64_t G = (int64_t)K.M * K.M * K.M, Gc = (int64_t)K.M * K.M * (K.M / 2 + 1);
    const int ch = fft_chunk(K.M);
    for (const BucketChunk& C : K.chunks) {
        if (slots <= 0) break;
        const int n = std::min(slots, C.slots) * ngrid;
        slots -= C.slots;
        for (int off = 0; off < n;) {
            const int b = fft_batch(n - off, ch);
            auto it = K.r2c.find(b);
            if (it == K.r2c.end()) return JT_ECUDA;   // bucket_ensure made every size a pass uses
            if (cufftExecR2C(it->second, C.rho + off * G, (cufftComplex*)(C.rho_k + off * Gc)) != CUFFT_SUCCESS)
                return JT_ECUDA;
            off += b;
        }
    }
    return JT_OK;
}

// the 3 ngrid force grids of the pass's first `slots` slots, chunk by chunk
int exec_c2r(Bucket& K, int slots, int ngrid)
{
    const int64_t G = (int64_t)K.M * K.M * K.M, Gc = (int64_t)K.M * K.M * (K.M / 2 + 1);
    const int ch = fft_chunk(K.M);
    for (const BucketChunk& C : K.chunks) {
        if (slots <= 0) break;
        const int n = std::min(slots, C.slots) * 3 * ngrid;
        slots -= C.slots;
        for (int off = 0; off < n;) {
            const int b = fft_batch(n - off, ch);
            auto it = K.c2r.find(b);
            if (it == K.c2r.end()) return JT_ECUDA;
            if (cufftExecC2R(it->second, (cufftComplex*)(C.force_k + off * Gc), C.force + off * G) != CUFFT_SUCCESS)
                return JT_ECUDA;
            off += b;
        }
    }
    return JT_OK;
}

template <class T>
size_t put(std::vector<unsigned char>& buf, const std::vector<T>& v)
{
    size_t off = (buf.size() + 15) & ~(size_t)15;
    buf.resize(off + sizeof(T) * v.size());
    if (!v.empty()) std::memcpy(buf.data() + off, v.data(), sizeof(T) * v.size());
    return off;
}

// Size the scratch pools for the listed boxes, lay out their segments and
// boxes, and upload every table in one copy.
int build_plan(jt_batch* B, const std::vector<int>& ids, const jt_box_step* steps, Plan& P)
{
    P = Plan();
    P.ids = ids;
    const int nb = (int)ids.size();
    const int ST = jt_sort_tile_size();
    int64_t nodes = 0, parts = 0, stiles = 0;
    int nseg = 0;
    for (int k = 0; k < nb; k++) {
        jt_box_state* b = B->boxes[ids[k]];
        for (int s = 0; s < 2; s++) {
            int64_t n = b->n[s];
            if (n == 0) continue;
            nodes += 2 * n - 1;
            parts += n;
            stiles += (n + ST - 1) / ST;
            nseg++;
        }
    }
    bool grew = false;
    JT_TRY(B->child.ensure(nodes, &grew)); JT_TRY(B->parent.ensure(nodes, &grew));
    JT_TRY(B->range.ensure(parts, &grew)); JT_TRY(B->flag.ensure(parts, &grew));
    JT_TRY(B->com.ensure(nodes, &grew)); JT_TRY(B->bmin.ensure(nodes, &grew));
    JT_TRY(B->bmax.ensure(nodes, &grew)); JT_TRY(B->quad0.ensure(nodes, &grew));
    JT_TRY(B->quad1.ensure(nodes, &grew));
    JT_TRY(B->m30.ensure(parts, &grew)); JT_TRY(B->vals.ensure(parts, &grew));
    JT_TRY(B->vals_alt.ensure(parts, &grew)); JT_TRY(B->keys_alt.ensure(parts, &grew));
    JT_TRY(B->hist.ensure((size_t)nseg * 4 * 256, &grew));
    JT_TRY(B->status.ensure((size_t)stiles * 4 * 256, &grew));
    JT_TRY(B->tickets.ensure(4, &grew));
    for (int k = 0; k < nb; k++) P.by_M[B->boxes[ids[k]]->M].push_back(k);
    std::vector<int> slot(nb);
    for (auto& kv : P.by_M) {
        int q = 0;
        for (int k : kv.second) {
            slot[k] = q;
            q += B->boxes[ids[k]]->ytab ? 2 : 1;
        }
        P.nslots[kv.first] = q;
    }
    for (auto& kv : P.nslots) JT_TRY(bucket_ensure(B, B->buckets[kv.first], kv.first, kv.second));
    if (B->fft_dirty || B->fftws.cap < B->fft_need) {
        bool ws_grew = false;
        JT_TRY(B->fftws.ensure(B->fft_need, &ws_grew));
        if (ws_grew) B->gen++;
        for (auto& kv : B->buckets) {
            for (auto& q : kv.second.r2c)
                if (cufftSetWorkArea(q.second, B->fftws.p) != CUFFT_SUCCESS) return JT_ECUDA;
            for (auto& q : kv.second.c2r)
                if (cufftSetWorkArea(q.second, B->fftws.p) != CUFFT_SUCCESS) return JT_ECUDA;
        }
        B->fft_dirty = false;
    }

    int64_t o_node = 0, o_part = 0, o_tile = 0;
    P.pprefix.push_back(0); P.iprefix.push_back(0); P.tprefix.push_back(0); P.gprefix.push_back(0);
    P.ptprefix.push_back(0); P.kprefix.push_back(0); P.cprefix.push_back(0); P.zprefix.push_back(0);
    P.cells = cells_enabled();
    P.bx.resize(nb);
    for (int k = 0; k < nb; k++) {
        jt_box_state* b = B->boxes[ids[k]];
        const jt_config& c = b->cfg;
        const int M = b->M;
        jt_box_dev& d = P.bx[k];
        std::memset(&d, 0, sizeof(d));
        d.L = (float)c.box_L;
        d.halfL = (float)(c.box_L / 2.0);
        d.box_half = (float)(c.box_L / 2.0);
        d.h_inv = (float)(M / c.box_L);
        const double rcut = jt_short_cut(c);
        d.rc2 = (float)(rcut * rcut);
        d.eps2 = (float)(c.softening * c.softening);
        d.c = (float)(1.0 / (2.0 * c.r_s));
        d.theta2 = (float)(c.theta * c.theta);
        d.mass[0] = b->mass[0];
        d.mass[1] = b->mass[1];
        d.kick_drag = steps ? steps[k].drag : 0.0f;
        d.dt = steps ? steps[k].dt : 0.0f;
        d.M = M;
        d.order = b->order;
        d.ngrid = b->ngrid;
        d.T = jt_pm_tile_edge(M);
        d.tile_shift = tile_shift_of(M);
        d.ntiles = (M / d.T) * (M / d.T) * (M / d.T);
        P.maxT = std::max(P.maxT, d.T);
        P.minT = std::min(P.minT, d.T);
        Bucket& K = B->buckets[M];
        const int q = slot[k];
        const int64_t G = (int64_t)M * M * M, Gc = (int64_t)M * M * (M / 2 + 1);
        int qi = 0;
        const BucketChunk& C = K.locate(q, &qi);
        d.rho = C.rho + (size_t)qi * b->ngrid * G;
        d.rho_k = C.rho_k + (size_t)qi * b->ngrid * Gc;
        d.force_k = C.force_k + (size_t)qi * 3 * b->ngrid * Gc;
        d.force = C.force + (size_t)qi * 3 * b->ngrid * G;
        d.tabs = b->tabs;
        d.ranges = C.ranges + (size_t)qi * d.ntiles;
        // the deposit flushes its tiles with 16-byte reductions
        if (reinterpret_cast<uintptr_t>(d.rho) & 15) return JT_ECUDA;
        if (b->ytab) {
            // the unsigned source's grids take the next slot (in this chunk
            // or the next)
            int si = 0;
            const BucketChunk& Cs = K.locate(q + 1, &si);
            d.rho_s = Cs.rho + (size_t)si * b->ngrid * G;
            d.rho_s_k = Cs.rho_k + (size_t)si * b->ngrid * Gc;
            d.force_s_k = Cs.force_k + (size_t)si * 3 * b->ngrid * Gc;
            d.force_s = Cs.force + (size_t)si * 3 * b->ngrid * G;
            d.ytab = b->ytab;
            d.ky2 = (float)(b->kappa * b->kappa);
            d.yfac = (float)std::exp(-b->kappa * b->kappa * c.r_s * c.r_s);
            P.screened = true;
        }
        d.seg[0] = d.seg[1] = -1;
        // near-field cells of side L / nb >= r_cut (1e-4 margin against
        // binning round-off); fewer than 3 per axis: tree walk only
        d.nb = 0;
        d.cbase = P.cprefix.back();
        if (P.cells && rcut > 0.0) {
            const double q = c.box_L / (rcut * 1.0001);
            int nbc = q >= 256.0 ? 256 : (int)q;
            if (nbc >= 3) d.nb = nbc;
            if (d.nb && b->cell_nb >= 3 && b->cell_nb < d.nb) d.nb = b->cell_nb;   // timed (tune_cells)
        }
        // a widened cut scales every neighbourhood's count by (cut / r_cut)^3,
        // and cells wider than the default by (default nb / nb)^3
        {
            const double w = rcut / c.r_cut;
            const double q = d.nb ? c.box_L / (rcut * 1.0001) : 0.0;
            const double v = d.nb ? std::min(256.0, std::floor(q)) / d.nb : 1.0;
            d.cell_kmax = (int)std::min(1.0e6, JT_CELL_KMAX * std::max(1.0, w * w * w) * v * v * v);
        }
        d.cell_inv = d.nb ? (float)(d.nb / c.box_L) : 0.0f;
        P.cprefix.push_back(P.cprefix.back() + (int64_t)d.nb * d.nb * d.nb);
        for (int s = 0; s < 2; s++) {
            const int64_t n = b->n[s];
            if (n == 0) continue;
            jt_seg_dev g;
            std::memset(&g, 0, sizeof(g));
            g.n = n;
            g.box = k;
            g.species = s;
            g.tree.n = n;
            g.tree.child = B->child.p + o_node;
            g.tree.parent = B->parent.p + o_node;
            g.tree.com = B->com.p + o_node;
            g.tree.bmin = B->bmin.p + o_node;
            g.tree.bmax = B->bmax.p + o_node;
            g.tree.quad0 = B->quad0.p + o_node;
            g.tree.quad1 = B->quad1.p + o_node;
            g.tree.range = B->range.p + o_part;
            g.tree.flag = B->flag.p + o_part;
            g.tree.m30 = B->m30.p + o_part;
            g.tree.tie = nullptr;   // Karras ties broken by sorted position
            g.vals = B->vals.p + o_part;
            g.vals_alt = B->vals_alt.p + o_part;
            g.keys_alt = B->keys_alt.p + o_part;
            g.hist = B->hist.p + (size_t)P.pre.size() * 4 * 256;
            g.status = B->status.p + (size_t)o_tile * 4 * 256;
            d.seg[s] = (int)P.pre.size();
            jt_seg_dev pre = g, post = g;
            pre.pos = b->pos[s]; pre.vel = b->vel[s]; pre.acc = b->acc[s];
            pre.pos_b = b->pos_b[s]; pre.vel_b = b->vel_b[s]; pre.id = b->id[s]; pre.id_b = b->id_b[s];
            post.pos = b->pos_b[s]; post.vel = b->vel_b[s]; post.acc = b->acc[s];
            post.pos_b = b->pos[s]; post.vel_b = b->vel[s]; post.id = b->id_b[s]; post.id_b = b->id[s];
            P.pre.push_back(pre);
            P.post.push_back(post);
            const int64_t t = (n + ST - 1) / ST;
            o_node += 2 * n - 1;
            o_part += n;
            o_tile += t;
            P.pprefix.push_back(P.pprefix.back() + n);
            P.iprefix.push_back(P.iprefix.back() + (n - 1));
            P.tprefix.push_back(P.tprefix.back() + t);
            P.gprefix.push_back(P.gprefix.back() + (n + 31) / 32);
        }
        P.ptprefix.push_back(P.ptprefix.back() + d.ntiles);
        // a fused bucket's boxes take the z kernel, the others k_b_kspace
        P.kprefix.push_back(P.kprefix.back() + (K.fused ? 0 : Gc));
        P.zprefix.push_back(P.zprefix.back() + (K.fused ? jt_zfft_tiles(M) : 0));
        if (K.fused) P.zsizes |= M == 512 ? 1 : 2;
    }
    P.npart = P.pprefix.back();
    P.ninternal = P.iprefix.back();
    P.nsorttiles = P.tprefix.back();
    P.ngroups = P.gprefix.back();
    P.npmtiles = P.ptprefix.back();
    P.nmodes = P.kprefix.back();
    P.nztiles = P.zprefix.back();
    P.ncells = P.cprefix.back();
    if (P.cells) {
        JT_TRY(B->ccount.ensure((size_t)std::max<int64_t>(P.ncells, 1), &grew));
        JT_TRY(B->cstart.ensure((size_t)P.ncells + 1, &grew));
        JT_TRY(B->cbsum.ensure((size_t)jt_cell_scan_blocks(P.ncells) + 1, &grew));
        JT_TRY(B->ccell.ensure((size_t)std::max<int64_t>(P.npart, 1), &grew));
        JT_TRY(B->cslot.ensure((size_t)std::max<int64_t>(P.npart, 1), &grew));
        JT_TRY(B->cpos.ensure((size_t)std::max<int64_t>(P.npart, 1), &grew));
        JT_TRY(B->cid.ensure((size_t)std::max<int64_t>(P.npart, 1), &grew));
        JT_TRY(B->tflag.ensure((size_t)std::max<int64_t>(P.npart, 1), &grew));
        JT_TRY(B->csegflag.ensure((size_t)std::max<int>(nseg, 1), &grew));
    }
    if (!P.screened) JT_TRY(B->pmacc.ensure((size_t)B->ngrid * std::max<int64_t>(P.npart, 1), &grew));

    if (grew) B->gen++;
    std::vector<unsigned char> buf;
    size_t o_pre = put(buf, P.pre), o_post = put(buf, P.post), o_bx = put(buf, P.bx);
    size_t o_pp = put(buf, P.pprefix), o_ip = put(buf, P.iprefix), o_tp = put(buf, P.tprefix);
    size_t o_gp = put(buf, P.gprefix), o_ptp = put(buf, P.ptprefix), o_kp = put(buf, P.kprefix);
    size_t o_cp = put(buf, P.cprefix), o_zp = put(buf, P.zprefix);
    JT_TRY(B->desc.ensure(buf.size(), &grew));
    // the previous upload may still read the staging buffer
    JT_CU(cudaEventSynchronize(B->desc_done));
    if (buf.size() > B->hdesc_cap) {
        if (B->hdesc) cudaFreeHost(B->hdesc);
        B->hdesc = nullptr;
        B->hdesc_cap = 0;
        if (cudaMallocHost((void**)&B->hdesc, buf.size() * 2) != cudaSuccess) return JT_ENOMEM;
        B->hdesc_cap = buf.size() * 2;
    }
    std::memcpy(B->hdesc, buf.data(), buf.size());
    JT_CU(cudaMemcpyAsync(B->desc.p, B->hdesc, buf.size(), cudaMemcpyHostToDevice, B->st));
    JT_CU(cudaEventRecord(B->desc_done, B->st));
    unsigned char* d = B->desc.p;
    P.d_pre = (const jt_seg_dev*)(d + o_pre);
    P.d_post = (const jt_seg_dev*)(d + o_post);
    P.d_bx = (const jt_box_dev*)(d + o_bx);
    P.d_pp = (const int64_t*)(d + o_pp);
    P.d_ip = (const int64_t*)(d + o_ip);
    P.d_tp = (const int64_t*)(d + o_tp);
    P.d_gp = (const int64_t*)(d + o_gp);
    P.d_ptp = (const int64_t*)(d + o_ptp);
    P.d_kp = (const int64_t*)(d + o_kp);
    P.d_cp = (const int64_t*)(d + o_cp);
    P.d_zp = (const int64_t*)(d + o_zp);
    P.table_bytes = buf.size();
    return JT_OK;
}

// The cell walk's cost depends on how a cell's targets fill batches of 32
// (a lattice whose points per cell are a whole number per axis fills them
// evenly), which no model of the mean count predicts: the first force-only
// pass of a box of kCellTuneMin particles or more, alone in its pass, times
// the cell walk at every nb from the default (side >= cut) down to 0.8 of it
// (the faster of two runs each) and keeps the fastest for the box (nb with
// targets flagged for the tree walk are not taken: they would time less
// work).  2x224^3 at cut 6 r_s: 68 -> 56 cells per axis (4 lattice points,
// 128 particles), cell walk 5 % faster.  JT_CELL_TUNE=0 in the environment
// (read once) keeps the default.
constexpr int64_t kCellTuneMin = (int64_t)1 << 22;

std::mutex g_cell_tune_mu;
std::string g_cell_tune_text;   // one entry per timed box (jt_cell_tuning_text)

int tune_cells(jt_batch* B, Plan& P, int nseg, int parts, const float4* pmacc)
{
    jt_box_state* bs = B->boxes[P.ids[0]];
    jt_box_dev& d = P.bx[0];
    if (!B->cell_tune || bs->cell_nb != 0 || d.nb < 8 || bs->n[0] + bs->n[1] < kCellTuneMin || P.screened ||
        nseg > 2)
        return JT_OK;
    static const bool off = [] {
        const char* e = std::getenv("JT_CELL_TUNE");
        return e && std::atoi(e) == 0;
    }();
    if (off) return JT_OK;   // JT_CELL_TUNE=0: the default cell count
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(B->st, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return JT_OK;
    cudaStream_t st = B->st;
    const int nmax = d.nb, kmax0 = d.cell_kmax, nmin = std::max(3, (int)std::ceil(0.8 * nmax));
    jt_cell_bufs cb = {B->ccount.p, B->cstart.p, B->cbsum.p, B->ccell.p, B->cslot.p,
                       B->cpos.p, B->cid.p, B->tflag.p, B->csegflag.p};
    cudaEvent_t e0, e1;
    JT_CU(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return JT_ECUDA;
    }
    auto set_nb = [&](int nb) -> int {
        const double v = (double)nmax / nb;
        d.nb = nb;
        d.cell_inv = (float)(nb / (double)d.L);
        d.cell_kmax = (int)std::min(1.0e6, kmax0 * v * v * v);
        P.cprefix[1] = (int64_t)nb * nb * nb;
        P.ncells = P.cprefix[1];
        if (cudaMemcpyAsync((void*)P.d_bx, &d, sizeof(jt_box_dev), cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync((void*)(P.d_cp + 1), &P.cprefix[1], sizeof(int64_t), cudaMemcpyHostToDevice, st) !=
                cudaSuccess)
            return JT_ECUDA;
        return JT_OK;
    };
    int r = JT_OK, best = nmax;
    float best_ms = 0.f;
    for (int nb = nmax; nb >= nmin && r == JT_OK; nb--) {
        r = set_nb(nb);
        // two runs, the faster one counts (candidates a few % apart)
        float ms = 0.f;
        int flag[2] = {0, 0};
        for (int rep = 0; rep < 2 && r == JT_OK; rep++) {
            r = jt_b_cells(P.d_post, P.d_bx, P.d_pp, nseg, P.npart, P.d_cp, 1, P.ncells, cb, B->order, B->ngrid,
                           parts, 0.0f, nullptr, B->d_err, st, e0, e1, false, pmacc, false);
            if (r == JT_OK && (cudaMemcpyAsync(flag, B->csegflag.p, sizeof(int) * (size_t)nseg,
                                               cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                               cudaStreamSynchronize(st) != cudaSuccess))
                r = JT_ECUDA;
            float m = 0.f;
            if (r == JT_OK && cudaEventElapsedTime(&m, e0, e1) != cudaSuccess) r = JT_ECUDA;
            if (r == JT_OK && (rep == 0 || m < ms)) ms = m;
        }
        if (r != JT_OK) break;
        if (nb == nmax) {
            best_ms = ms;
            if (flag[0] || flag[1]) break;   // crowded at the default already: keep it
        } else if (!flag[0] && !flag[1] && ms < best_ms) {
            best = nb;
            best_ms = ms;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (r != JT_OK) return r;
    bs->cell_nb = best;
    {
        std::lock_guard<std::mutex> lock(g_cell_tune_mu);
        if (g_cell_tune_text.size() < 4096)
            g_cell_tune_text += "cells " + std::to_string(bs->n[0] + bs->n[1]) + " particles: " +
                                std::to_string(nmax) + " -> " + std::to_string(best) + " per axis; ";
    }
    return set_nb(best);
}

// One force pass over the plan's boxes; afterwards every box's state sits in
// its former b-buffers (pointers swapped here and in the plan).
int force_pass(jt_batch* B, Plan& P, int parts, float kick_frac)
{
    cudaStream_t st = B->st;
    const int nseg = (int)P.pre.size(), nbox = (int)P.bx.size();
    cudaEventRecord(B->ev[0], st);
    JT_CU(cudaMemsetAsync(B->hist.p, 0, sizeof(uint32_t) * (size_t)nseg * 4 * 256, st));
    JT_CU(cudaMemsetAsync(B->status.p, 0, sizeof(uint32_t) * (size_t)P.nsorttiles * 4 * 256, st));
    JT_CU(cudaMemsetAsync(B->tickets.p, 0, sizeof(uint32_t) * 4, st));
    JT_TRY(jt_b_sort_reorder(P.d_pre, P.d_bx, nseg, P.d_pp, P.npart, P.d_tp, P.nsorttiles, B->tickets.p,
                             B->d_err, st));
    cudaEventRecord(B->ev[1], st);
    // with the cell walk the trees are built after it, for the segments whose
    // particles it flagged (none for uniform data)
    if (!P.cells) jt_b_build_trees(P.d_post, P.d_bx, nseg, P.d_ip, P.ninternal, P.d_pp, P.npart, st);
    cudaEventRecord(B->ev[2], st);
    for (auto& kv : P.nslots) {
        const int64_t M = kv.first, G = M * M * M;
        int left = kv.second;
        for (const BucketChunk& C : B->buckets[kv.first].chunks) {
            if (left <= 0) break;
            const int u = std::min(left, C.slots);
            JT_CU(cudaMemsetAsync(C.rho, 0, sizeof(float) * u * B->ngrid * G, st));
            left -= u;
        }
    }
    jt_b_tile_ranges(P.d_post, P.d_bx, P.d_ptp, nbox, P.npmtiles, st);
    const bool t16 = P.minT == 16 && P.maxT == 16;
    JT_TRY(jt_b_deposit(P.d_post, P.d_bx, P.d_ptp, nbox, P.npmtiles, B->order, B->ngrid, P.maxT, st, 0, t16));
    if (P.screened)
        JT_TRY(jt_b_deposit(P.d_post, P.d_bx, P.d_ptp, nbox, P.npmtiles, B->order, B->ngrid, P.maxT, st, 1, t16));
    cudaEventRecord(B->ev[3], st);
    for (auto& kv : P.nslots) {
        Bucket& K = B->buckets[kv.first];
        JT_TRY(exec_r2c(K, kv.second, B->ngrid));
    }
    cudaEventRecord(B->ev[4], st);
    jt_b_kspace(P.d_bx, P.d_kp, nbox, P.nmodes, B->ngrid == 2, B->k_min, st);
    JT_TRY(jt_b_zfft_kspace(P.d_bx, P.d_zp, nbox, P.nztiles, B->ngrid == 2, B->k_min, 0, P.zsizes, st));
    if (P.screened)
        JT_TRY(jt_b_zfft_kspace(P.d_bx, P.d_zp, nbox, P.nztiles, B->ngrid == 2, B->k_min, 1, P.zsizes, st));
    cudaEventRecord(B->ev[5], st);
    for (auto& kv : P.nslots) {
        Bucket& K = B->buckets[kv.first];
        JT_TRY(exec_c2r(K, kv.second, B->ngrid));
    }
    cudaEventRecord(B->ev[6], st);
    // PM interpolation of every particle from shared-memory tiles (a pass with
    // a screened box interpolates inside the walks: it has two sets of grids)
    const float4* pmacc = nullptr;
    if (!P.screened && (parts & JT_PART_PM) && P.npart > 0) {
        JT_TRY(jt_b_interp(P.d_post, P.d_bx, P.d_ptp, P.d_pp, nbox, P.npmtiles, B->order, B->ngrid, P.maxT,
                           P.npart, B->pmacc.p, st, t16));
        pmacc = B->pmacc.p;
        B->tm.launches += 1;
    }
    cudaEventRecord(B->ev[10], st);
    jt_tree_dev pool = {};
    pool.child = B->child.p;
    pool.range = B->range.p;
    pool.parent = B->parent.p;
    pool.flag = B->flag.p;
    pool.com = B->com.p;
    pool.bmin = B->bmin.p;
    pool.bmax = B->bmax.p;
    pool.quad0 = B->quad0.p;
    pool.quad1 = B->quad1.p;
    pool.m30 = B->m30.p;
    const unsigned char* tflag = nullptr;
    if (!P.cells) {
        cudaEventRecord(B->ev[8], st);
        cudaEventRecord(B->ev[9], st);
    } else {
        if (kick_frac == 0.0f && nbox == 1 && P.ncells > 0 && (parts & JT_PART_SHORT))
            JT_TRY(tune_cells(B, P, nseg, parts, pmacc));
        jt_cell_bufs cb = {B->ccount.p, B->cstart.p, B->cbsum.p, B->ccell.p, B->cslot.p,
                           B->cpos.p, B->cid.p, B->tflag.p, B->csegflag.p};
        JT_TRY(jt_b_cells(P.d_post, P.d_bx, P.d_pp, nseg, P.npart, P.d_cp, nbox, P.ncells, cb, B->order,
                          B->ngrid, parts, kick_frac, B->d_stats, B->d_err, st, B->ev[8], B->ev[9],
                          P.screened, pmacc, B->counters));
        tflag = B->tflag.p;
        jt_b_build_trees(P.d_post, P.d_bx, nseg, P.d_ip, P.ninternal, P.d_pp, P.npart, st, B->csegflag.p);
        B->tm.launches += P.npart > 0 ? (P.ncells > 0 ? 6 : 1) : 0;
    }
    JT_TRY(jt_b_walk(P.d_post, P.d_bx, P.d_gp, nseg, P.ngroups, pool, B->order, B->ngrid, parts,
                     kick_frac, B->d_stats, B->d_err, st, P.d_pp, tflag, P.screened,
                     tflag ? B->csegflag.p : nullptr, pmacc, P.npart));
    cudaEventRecord(B->ev[7], st);
    B->pending = true;
    B->tm.launches += (P.npart > 0 ? 8 : 0) + (P.ninternal > 0 ? 1 : 0) + (P.npart > 0 ? 1 : 0) +
                      (P.npmtiles > 0 ? (P.screened ? 3 : 2) : 0) + (P.nmodes > 0 ? 1 : 0) +
                      (P.nztiles > 0 ? (P.screened ? 2 : 1) * ((P.zsizes & 1) + ((P.zsizes >> 1) & 1)) : 0) +
                      (P.ngroups > 0 ? 1 : 0);
    for (int id : P.ids) {
        jt_box_state* b = B->boxes[id];
        for (int s = 0; s < 2; s++) {
            std::swap(b->pos[s], b->pos_b[s]);
            std::swap(b->vel[s], b->vel_b[s]);
            std::swap(b->id[s], b->id_b[s]);
        }
        b->acc_valid = parts == JT_PART_ALL;
    }
    std::swap(P.pre, P.post);
    std::swap(P.d_pre, P.d_post);
    return cudaGetLastError() == cudaSuccess ? JT_OK : JT_ECUDA;
}

int finish(jt_batch* B)
{
    unsigned e = 0;
    unsigned long long v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    JT_CU(cudaMemcpyAsync(&e, B->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost, B->st));
    JT_CU(cudaMemcpyAsync(v, B->d_stats, sizeof(v), cudaMemcpyDeviceToHost, B->st));
    JT_CU(cudaStreamSynchronize(B->st));
    if (e) {
        for (jt_box_state* b : B->boxes)
            if (b) b->acc_valid = false;
        cudaMemsetAsync(B->d_err, 0, sizeof(unsigned), B->st);
        cudaMemsetAsync(B->d_stats, 0, sizeof(v), B->st);
        cudaStreamSynchronize(B->st);
        B->pending = false;
        return (e & JT_ERRBIT_LOOKBACK) ? JT_ETIMEDOUT : JT_EOVERFLOW;
    }
    if (B->pending) {
        B->tm.sort_ms += elapsed(B->ev[0], B->ev[1]);
        B->tm.tree_ms += elapsed(B->ev[1], B->ev[2]);
        B->tm.deposit_ms += elapsed(B->ev[2], B->ev[3]);
        B->tm.fft_ms += elapsed(B->ev[3], B->ev[6]);
        B->tm.kspace_ms += elapsed(B->ev[4], B->ev[5]);
        B->tm.walk_ms += elapsed(B->ev[6], B->ev[7]);
        B->tm.cellwalk_ms += elapsed(B->ev[8], B->ev[9]);
        B->tm.interp_ms += elapsed(B->ev[6], B->ev[10]);
        B->pending = false;
    }
    B->tm.pair_interactions += (int64_t)v[0];
    B->tm.node_interactions += (int64_t)v[1];
    B->tm.candidates += (int64_t)v[2];
    B->tm.interactions += (int64_t)(v[0] + v[1]);
    for (int i = 0; i < 4; i++) B->phase[i] += (int64_t)v[3 + i];
    JT_CU(cudaMemsetAsync(B->d_stats, 0, sizeof(v), B->st));
    return JT_OK;
}

int valid_ids(jt_batch* B, const int* ids, int n, std::vector<int>& out)
{
    out.clear();
    if (!ids || n <= 0) return JT_EINVAL;
    std::vector<char> seen(B->boxes.size(), 0);
    for (int k = 0; k < n; k++) {
        int id = ids[k];
        if (id < 0 || id >= (int)B->boxes.size() || !B->boxes[id] || seen[id]) return JT_EINVAL;
        seen[id] = 1;
        out.push_back(id);
    }
    return JT_OK;
}

}  // namespace

double jt_short_cut(const jt_config& c)
{
    if (c.cut_tail_ppm <= 0 || !(c.r_s > 0.0)) return c.r_cut;
    // S(x) = erfc(x) + (2 / sqrt(pi)) x e^{-x^2} decreases monotonically:
    // bisection for S(x) = tol on [0, 8]
    const double tol = 1e-6 * c.cut_tail_ppm;
    auto S = [](double x) { return std::erfc(x) + 1.1283791670955126 * x * std::exp(-x * x); };
    double lo = 0.0, hi = 8.0;
    for (int it = 0; it < 80; it++) {
        const double mid = 0.5 * (lo + hi);
        if (S(mid) > tol) lo = mid; else hi = mid;
    }
    return std::max(c.r_cut, 2.0 * c.r_s * hi);
}

namespace {

int validate_box_config(const jt_config* c)
{
    auto pow2 = [](int m) { return m > 0 && (m & (m - 1)) == 0; };
    if (!c) return JT_EINVAL;
    if (c->mode != JT_ACCURATE || c->integrator != JT_KDK) return JT_EINVAL;
    if (!(c->box_L > 0.0) || !std::isfinite(c->box_L)) return JT_EINVAL;
    if (!pow2(c->pm_grid) || c->pm_grid < 8 || c->pm_grid > 1024) return JT_EINVAL;
    if (!(c->theta >= 0.0) || !std::isfinite(c->theta)) return JT_EINVAL;
    if (!(c->softening >= 0.0) || !std::isfinite(c->softening)) return JT_EINVAL;
    if (!(c->r_cut > 0.0) || c->r_cut >= 0.5 * c->box_L) return JT_EINVAL;
    if (!(c->r_s > 0.0) || !std::isfinite(c->r_s)) return JT_EINVAL;
    if (c->cut_tail_ppm < 0 || c->cut_tail_ppm >= 1000000) return JT_EINVAL;
    if (!(jt_short_cut(*c) < 0.5 * c->box_L)) return JT_EINVAL;
    if (!(c->mu >= 0.0) || !std::isfinite(c->mu)) return JT_EINVAL;
    if (!(c->G_mass_plus > 0.0) || !std::isfinite(c->G_mass_plus)) return JT_EINVAL;
    if (c->k_min < 0) return JT_EINVAL;
    if (c->pm_order != 0 && (c->pm_order < 2 || c->pm_order > 4)) return JT_EINVAL;
    if (c->pm_interlace < 0 || c->pm_interlace > 2) return JT_EINVAL;
    return JT_OK;
}

bool box_id_ok(jt_batch* B, int id) { return B && id >= 0 && id < (int)B->boxes.size() && B->boxes[id]; }

// AoS float3 out of a box (caller order of the species array).
int read_out(jt_batch* B, const float4* src, const int* id, int64_t n, float* dst, int mem)
{
    if (!dst || n == 0) return JT_OK;
    if (mem == JT_MEM_DEVICE) {
        jt_launch_aos_out(src, id, nullptr, n, dst, B->st);
        return JT_OK;
    }
    bool grew = false;
    JT_TRY(B->stage.ensure(3 * (size_t)n, &grew));
    jt_launch_aos_out(src, id, nullptr, n, B->stage.p, B->st);
    cudaError_t e = cudaMemcpyAsync(dst, B->stage.p, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, B->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(B->st);
    return e == cudaSuccess ? JT_OK : JT_ECUDA;
}

}  // namespace

void drop_graphs(jt_batch* B)
{
    for (auto& e : B->gc.exec)
        if (e) {
            cudaGraphExecDestroy(e);
            e = nullptr;
        }
    B->gc.ids.clear();
    B->gc.gen = ~0ull;
}

void swap_state(jt_batch* B, const std::vector<int>& v)
{
    for (int id : v) {
        jt_box_state* b = B->boxes[id];
        for (int s = 0; s < 2; s++) {
            std::swap(b->pos[s], b->pos_b[s]);
            std::swap(b->vel[s], b->vel_b[s]);
            std::swap(b->id[s], b->id_b[s]);
        }
    }
}

// Capture one KDK step of boxes v -- kick(dt/2), drift(dt), force pass with
// the closing kick(dt/2) fused into the walk -- as two CUDA graphs, one per
// parity of the ping-pong buffers (the reorder of every pass swaps them).
// The graphs read a private copy of the step's tables (gdesc), so other
// passes may rebuild the batch's own tables freely; any change of a device
// address the tables hold bumps B->gen and invalidates the graphs.
int capture_graphs(jt_batch* B, const std::vector<int>& v, const jt_box_step* steps)
{
    drop_graphs(B);
    Plan P;
    JT_TRY(build_plan(B, v, steps, P));
    bool grew = false;
    JT_TRY(B->gdesc.ensure(P.table_bytes, &grew));
    JT_CU(cudaMemcpyAsync(B->gdesc.p, B->desc.p, P.table_bytes, cudaMemcpyDeviceToDevice, B->st));
    auto rebase = [&](const void* p) -> const void* {
        return B->gdesc.p + ((const unsigned char*)p - B->desc.p);
    };
    P.d_pre = (const jt_seg_dev*)rebase(P.d_pre);
    P.d_post = (const jt_seg_dev*)rebase(P.d_post);
    P.d_bx = (const jt_box_dev*)rebase(P.d_bx);
    P.d_pp = (const int64_t*)rebase(P.d_pp);
    P.d_ip = (const int64_t*)rebase(P.d_ip);
    P.d_tp = (const int64_t*)rebase(P.d_tp);
    P.d_gp = (const int64_t*)rebase(P.d_gp);
    P.d_ptp = (const int64_t*)rebase(P.d_ptp);
    P.d_kp = (const int64_t*)rebase(P.d_kp);
    P.d_zp = (const int64_t*)rebase(P.d_zp);
    const jt_timings saved = B->tm;
    const jt_box_state* b0 = B->boxes[v[0]];
    const int sp0 = b0->n[0] > 0 ? 0 : 1;
    const float4* pre0 = b0->pos[sp0];
    int r = JT_OK;
    for (int parity = 0; parity < 2 && r == JT_OK; parity++) {
        if (cudaStreamBeginCapture(B->st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            r = JT_ECUDA;
            break;
        }
        jt_b_kick_drift(P.d_pre, P.d_bx, P.d_pp, (int)P.pre.size(), P.npart, 0.5f, 1.0f, B->st);
        int rf = force_pass(B, P, JT_PART_ALL, 0.5f);   // swaps the boxes' buffers and P
        cudaGraph_t g = nullptr;
        cudaError_t ec = cudaStreamEndCapture(B->st, &g);
        if (rf != JT_OK || ec != cudaSuccess || !g) {
            if (g) cudaGraphDestroy(g);
            r = rf != JT_OK ? rf : JT_ECUDA;
            break;
        }
        if (cudaGraphInstantiate(&B->gc.exec[parity], g, 0) != cudaSuccess) r = JT_ECUDA;
        cudaGraphDestroy(g);
    }
    const int64_t per_pass = B->tm.launches - saved.launches;
    B->tm = saved;
    B->pending = false;
    cudaGetLastError();
    // nothing ran during the captures: if they left the host pointers
    // swapped an odd number of times, swap them back
    if (b0->pos[sp0] != pre0) swap_state(B, v);
    if (r != JT_OK) {
        drop_graphs(B);
        return r;
    }
    B->gc.launches = per_pass / 2 + 1;   // the force pass and the kick-drift
    B->gc.ids = v;
    B->gc.gen = B->gen;
    B->gc.plan = P;
    B->gc.box0 = v[0];
    B->gc.sp0 = sp0;
    B->gc.pre0 = pre0;
    return JT_OK;
}

// ---------------------------------------------------------------- internal
int jtb_add_empty(jt_batch* B, const jt_config* cfg, int64_t n_p, int64_t n_m, int* box_id)
{
    if (!B || !box_id || n_p < 0 || n_m < 0 || n_p + n_m == 0) return JT_EINVAL;
    AllocScope scope(&B->actx);
    if (n_p >= (int64_t)1 << 30 || n_m >= (int64_t)1 << 30) return JT_EINVAL;
    JT_TRY(validate_box_config(cfg));
    const int order = box_order(*cfg), ngrid = box_ngrid(*cfg);
    bool empty = true;
    for (auto* b : B->boxes) empty = empty && !b;
    if (!empty && (order != B->order || ngrid != B->ngrid || cfg->k_min != B->k_min)) return JT_EINVAL;
    jt_box_state* b = new (std::nothrow) jt_box_state();
    if (!b) return JT_ENOMEM;
    b->cfg = *cfg;
    b->n[0] = n_p;
    b->n[1] = n_m;
    // per-particle masses: m+ = G_mass_plus, m- = mu m+ N+/N- (mu = M-/M+)
    double mp = cfg->G_mass_plus;
    double mm = n_m > 0 ? cfg->mu * mp * (double)n_p / (double)n_m : 0.0;
    if (n_p == 0) mm = cfg->mu * mp;
    b->mass[0] = (float)mp;
    b->mass[1] = (float)mm;
    b->M = cfg->pm_grid;
    b->order = order;
    b->ngrid = ngrid;
    int r = box_alloc(b);
    if (r != JT_OK) {
        box_release(b);
        delete b;
        return r;
    }
    int slot = -1;
    for (size_t k = 0; k < B->boxes.size(); k++)
        if (!B->boxes[k]) { slot = (int)k; break; }
    if (slot < 0) {
        slot = (int)B->boxes.size();
        B->boxes.push_back(nullptr);
    }
    B->boxes[slot] = b;
    B->gen++;
    B->order = order;
    B->ngrid = ngrid;
    B->k_min = cfg->k_min;
    *box_id = slot;
    return JT_OK;
}

jt_box_state* jtb_box(jt_batch* B, int box_id) { return box_id_ok(B, box_id) ? B->boxes[box_id] : nullptr; }

cudaStream_t jtb_stream(jt_batch* B) { return B ? B->st : nullptr; }

int jtb_force_pass(jt_batch* B, const int* ids, int n_ids, int parts, float kick_frac, const jt_box_step* steps)
{
    if (!B || parts < 1 || parts > 3) return JT_EINVAL;
    AllocScope scope(&B->actx);
    std::vector<int> v;
    JT_TRY(valid_ids(B, ids, n_ids, v));
    JT_TRY(build_plan(B, v, steps, B->plan));
    return force_pass(B, B->plan, parts, kick_frac);
}

int jtb_finish(jt_batch* B) { return B ? finish(B) : JT_EINVAL; }

void jtb_reset_timings(jt_batch* B)
{
    if (B) B->tm = jt_timings{};
}

jt_ckpt** jtb_ckpt_slot(jt_batch* B) { return &B->ckpt; }
int64_t jtb_phase(jt_batch* B, int i) { return B && i >= 0 && i < 4 ? B->phase[i] : 0; }

int jtb_set_accel(jt_batch* B, int box_id, const float* acc_p, const float* acc_m, int mem)
{
    if (!box_id_ok(B, box_id) || (mem != JT_MEM_HOST && mem != JT_MEM_DEVICE)) return JT_EINVAL;
    AllocScope scope(&B->actx);
    jt_box_state* b = B->boxes[box_id];
    const float* src[2] = {acc_p, acc_m};
    for (int s = 0; s < 2; s++) {
        const int64_t n = b->n[s];
        if (n == 0) continue;
        if (!src[s]) return JT_EINVAL;
        // accelerations are stored in the state's internal order: map the
        // caller's order through id (after an add, internal = caller order)
        const float* d = src[s];
        if (mem == JT_MEM_HOST) {
            bool grew = false;
            JT_TRY(B->stage.ensure(3 * (size_t)n, &grew));
            JT_CU(cudaMemcpyAsync(B->stage.p, src[s], sizeof(float) * 3 * n, cudaMemcpyHostToDevice, B->st));
            d = B->stage.p;
        }
        jt_launch_aos_in(d, n, b->acc[s], nullptr, B->st);
        JT_CU(cudaStreamSynchronize(B->st));
    }
    JT_CU(cudaGetLastError());
    b->acc_valid = true;
    return JT_OK;
}

int jtb_upload_async(jt_batch* B, int box_id, const float* const pos[2], const float* const vel[2],
                     const float* const acc[2])
{
    if (!box_id_ok(B, box_id)) return JT_EINVAL;
    AllocScope scope(&B->actx);
    jt_box_state* b = B->boxes[box_id];
    for (int s = 0; s < 2; s++) {
        const int64_t n = b->n[s];
        if (n == 0) continue;
        if (!pos[s] || (acc && !acc[s])) return JT_EINVAL;
        // the kernels read the pinned host arrays through their device
        // addresses (no staging buffer, no copy engine)
        jt_launch_host_in(pos[s], n, b->pos[s], b->id[s], B->st);
        if (vel && vel[s]) jt_launch_host_in(vel[s], n, b->vel[s], nullptr, B->st);
        else JT_CU(cudaMemsetAsync(b->vel[s], 0, sizeof(float4) * (size_t)n, B->st));
        if (acc) jt_launch_host_in(acc[s], n, b->acc[s], nullptr, B->st);
    }
    JT_CU(cudaGetLastError());
    b->acc_valid = acc != nullptr;
    return JT_OK;
}

int jtb_download_async(jt_batch* B, int box_id, float* const pos[2], float* const vel[2], float* const acc[2],
                       bool* acc_copied)
{
    if (!box_id_ok(B, box_id)) return JT_EINVAL;
    AllocScope scope(&B->actx);
    jt_box_state* b = B->boxes[box_id];
    const bool with_acc = acc != nullptr && b->acc_valid;
    for (int s = 0; s < 2; s++) {
        const int64_t n = b->n[s];
        if (n == 0) continue;
        // the kernels write the pinned host arrays through their device
        // addresses, in caller order; the inverse order goes into the
        // reorder's spare id buffer (rewritten by the next sort)
        int* inv = b->id_b[s];
        jt_launch_inverse(b->id[s], n, inv, B->st);
        if (pos[s]) jt_launch_host_out(b->pos[s], inv, n, pos[s], B->st);
        if (vel[s]) jt_launch_host_out(b->vel[s], inv, n, vel[s], B->st);
        if (with_acc && acc[s]) jt_launch_host_out(b->acc[s], inv, n, acc[s], B->st);
    }
    JT_CU(cudaGetLastError());
    if (acc_copied) *acc_copied = with_acc;
    return JT_OK;
}

int jtb_remove_async(jt_batch* B, int box_id)
{
    if (!box_id_ok(B, box_id)) return JT_EINVAL;
    AllocScope scope(&B->actx);
    box_release(B->boxes[box_id]);   // stream-ordered frees: after the work queued on the box
    B->gen++;
    delete B->boxes[box_id];
    B->boxes[box_id] = nullptr;
    return JT_OK;
}

int jtb_step_host(jt_batch* B, int box_id, float* const pos[2], float* const vel[2], float* const acc[2],
                  float dt, float drag)
{
    if (!box_id_ok(B, box_id) || !std::isfinite(dt) || !std::isfinite(drag)) return JT_EINVAL;
    AllocScope scope(&B->actx);
    jt_box_state* b = B->boxes[box_id];
    for (int s = 0; s < 2; s++)
        if (b->n[s] > 0 && (!pos[s] || !vel[s] || !acc[s])) return JT_EINVAL;
    bool grew = false;
    JT_TRY(B->io.ensure(9 * (size_t)(b->n[0] + b->n[1]), &grew));
    if (!B->io_side) {
        JT_CU(cudaStreamCreateWithFlags(&B->io_side, cudaStreamNonBlocking));
        JT_CU(cudaEventCreateWithFlags(&B->io_ev, cudaEventDisableTiming));
    }
    cudaStream_t st = B->st;
    B->tm = jt_timings{};
    cudaEvent_t t0, t1, k0, k1;
    cudaEventCreate(&t0); cudaEventCreate(&t1); cudaEventCreate(&k0); cudaEventCreate(&k1);
    cudaEventRecord(t0, st);
    float* io[2] = {B->io.p, B->io.p + 9 * (size_t)b->n[0]};
    int r = JT_OK;
    // upload in the order the kick and the drift need the arrays; the box
    // takes the caller's order (id = identity)
    for (int s = 0; s < 2 && r == JT_OK; s++) {
        const int64_t n = b->n[s];
        if (n == 0) continue;
        const size_t bytes = sizeof(float) * 3 * (size_t)n;
        if (cudaMemcpyAsync(io[s] + 6 * n, acc[s], bytes, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(io[s] + 3 * n, vel[s], bytes, cudaMemcpyHostToDevice, st) != cudaSuccess ||
            cudaMemcpyAsync(io[s], pos[s], bytes, cudaMemcpyHostToDevice, st) != cudaSuccess)
            r = JT_ECUDA;
        jt_launch_aos_in(io[s] + 6 * n, n, b->acc[s], nullptr, st);
        jt_launch_aos_in(io[s] + 3 * n, n, b->vel[s], nullptr, st);
        jt_launch_aos_in(io[s], n, b->pos[s], b->id[s], st);
        B->tm.launches += 3;
    }
    b->acc_valid = true;
    const jt_box_step step = {dt, drag};
    const std::vector<int> v(1, box_id);
    Plan& P = B->plan;
    if (r == JT_OK) r = build_plan(B, v, &step, P);
    double kd = 0.0;
    if (r == JT_OK) {
        cudaEventRecord(k0, st);
        jt_b_kick_drift(P.d_pre, P.d_bx, P.d_pp, (int)P.pre.size(), P.npart, 0.5f, 1.0f, st);
        cudaEventRecord(k1, st);
        B->tm.launches += 1;
        // the positions are final: pack them into their upload slots (still
        // in the caller's order) and copy them back while the forces run
        for (int s = 0; s < 2; s++)
            if (b->n[s] > 0) {
                jt_launch_aos_out(b->pos[s], b->id[s], nullptr, b->n[s], io[s], st);
                B->tm.launches += 1;
            }
        if (cudaEventRecord(B->io_ev, st) != cudaSuccess ||
            cudaStreamWaitEvent(B->io_side, B->io_ev, 0) != cudaSuccess)
            r = JT_ECUDA;
        for (int s = 0; s < 2 && r == JT_OK; s++)
            if (b->n[s] > 0 &&
                cudaMemcpyAsync(pos[s], io[s], sizeof(float) * 3 * (size_t)b->n[s], cudaMemcpyDeviceToHost,
                                B->io_side) != cudaSuccess)
                r = JT_ECUDA;
    }
    if (r == JT_OK) r = force_pass(B, P, JT_PART_ALL, 0.5f);
    if (r == JT_OK) {
        // velocities (closing half kick fused into the walk) and
        // accelerations, back to the caller's order
        for (int s = 0; s < 2 && r == JT_OK; s++) {
            const int64_t n = b->n[s];
            if (n == 0) continue;
            const size_t bytes = sizeof(float) * 3 * (size_t)n;
            jt_launch_aos_out(b->vel[s], b->id[s], nullptr, n, io[s] + 3 * n, st);
            jt_launch_aos_out(b->acc[s], b->id[s], nullptr, n, io[s] + 6 * n, st);
            B->tm.launches += 2;
            if (cudaMemcpyAsync(vel[s], io[s] + 3 * n, bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
                cudaMemcpyAsync(acc[s], io[s] + 6 * n, bytes, cudaMemcpyDeviceToHost, st) != cudaSuccess)
                r = JT_ECUDA;
        }
        kd = elapsed(k0, k1);
        if (r == JT_OK) r = finish(B);
    }
    cudaEventRecord(t1, st);
    if (cudaStreamSynchronize(st) != cudaSuccess && r == JT_OK) r = JT_ECUDA;
    if (cudaStreamSynchronize(B->io_side) != cudaSuccess && r == JT_OK) r = JT_ECUDA;
    if (r == JT_OK) {
        B->tm.total_ms = elapsed(t0, t1);
        B->tm.kick_drift_ms = kd;
    } else {
        b->acc_valid = false;
    }
    cudaEventDestroy(t0); cudaEventDestroy(t1); cudaEventDestroy(k0); cudaEventDestroy(k1);
    return r;
}

// ---------------------------------------------------------------- C ABI
extern "C" {

int jt_batch_create(jt_batch** out)
{
    if (!out) return JT_EINVAL;
    *out = nullptr;
    jt_batch* B = new (std::nothrow) jt_batch();
    if (!B) return JT_ENOMEM;
    if (cudaGetDevice(&B->device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&B->st, cudaStreamNonBlocking) != cudaSuccess) {
        delete B;
        return JT_ECUDA;
    }
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = B->device;
    if (cudaMemPoolCreate(&B->actx.pool, &props) != cudaSuccess) {
        cudaStreamDestroy(B->st);
        delete B;
        return JT_ECUDA;
    }
    // keep freed blocks for reuse (jt_batch_trim returns them to the device)
    uint64_t keep = ~(uint64_t)0;
    cudaMemPoolSetAttribute(B->actx.pool, cudaMemPoolAttrReleaseThreshold, &keep);
    B->actx.st = B->st;
    if (const char* e = getenv("JT_COUNTERS")) B->counters = atoi(e) != 0;
    for (auto& e : B->ev) cudaEventCreate(&e);
    cudaEventCreateWithFlags(&B->desc_done, cudaEventDisableTiming);
    if (cudaMalloc(&B->d_err, sizeof(unsigned)) != cudaSuccess ||
        cudaMalloc(&B->d_stats, 8 * sizeof(unsigned long long)) != cudaSuccess) {
        jt_batch_destroy(B);
        return JT_ENOMEM;
    }
    cudaMemset(B->d_err, 0, sizeof(unsigned));
    cudaMemset(B->d_stats, 0, 8 * sizeof(unsigned long long));
    *out = B;
    return JT_OK;
}

void jt_batch_destroy(jt_batch* B)
{
    if (!B) return;
    AllocScope scope(&B->actx);
    jt_ckpt_release(B->ckpt);
    if (B->st) cudaStreamSynchronize(B->st);
    for (auto* b : B->boxes)
        if (b) { box_release(b); delete b; }
    B->child.release(); B->range.release(); B->parent.release(); B->flag.release();
    B->com.release(); B->bmin.release(); B->bmax.release(); B->quad0.release(); B->quad1.release();
    B->ccount.release(); B->cstart.release(); B->cbsum.release(); B->ccell.release(); B->cslot.release();
    B->csegflag.release();
    B->cpos.release(); B->cid.release(); B->tflag.release(); B->pmacc.release();
    B->m30.release(); B->vals.release(); B->vals_alt.release(); B->keys_alt.release();
    B->hist.release(); B->status.release(); B->tickets.release(); B->desc.release();
    drop_graphs(B);
    B->gdesc.release();
    for (auto& kv : B->buckets) kv.second.release();
    B->fftws.release();
    B->stage.release();
    B->io.release();
    if (B->io_side) {
        cudaStreamSynchronize(B->io_side);
        cudaStreamDestroy(B->io_side);
    }
    if (B->io_ev) cudaEventDestroy(B->io_ev);
    if (B->hdesc) cudaFreeHost(B->hdesc);
    if (B->d_err) cudaFree(B->d_err);
    if (B->d_stats) cudaFree(B->d_stats);
    for (auto& e : B->ev)
        if (e) cudaEventDestroy(e);
    if (B->desc_done) cudaEventDestroy(B->desc_done);
    if (B->st) cudaStreamSynchronize(B->st);
    if (B->actx.pool) cudaMemPoolDestroy(B->actx.pool);
    if (B->st) cudaStreamDestroy(B->st);
    delete B;
}

int jt_batch_add(jt_batch* B, const jt_config* cfg, const float* pos_p, const float* vel_p, size_t n_p,
                 const float* pos_m, const float* vel_m, size_t n_m, int mem, int* box_id)
{
    if (!B || !cfg || !box_id || (mem != JT_MEM_HOST && mem != JT_MEM_DEVICE)) return JT_EINVAL;
    AllocScope scope(&B->actx);
    if ((n_p && !pos_p) || (n_m && !pos_m)) return JT_EINVAL;
    if (n_p >= (size_t)1 << 30 || n_m >= (size_t)1 << 30) return JT_EINVAL;
    int id = -1;
    JT_TRY(jtb_add_empty(B, cfg, (int64_t)n_p, (int64_t)n_m, &id));
    jt_box_state* b = B->boxes[id];
    const float* pp[2] = {pos_p, pos_m};
    const float* vv[2] = {vel_p, vel_m};
    int r = JT_OK;
    float* stage = nullptr;
    if (mem == JT_MEM_HOST) {
        bool grew = false;
        r = B->stage.ensure(3 * std::max(n_p, n_m), &grew);
        stage = B->stage.p;
    }
    for (int s = 0; s < 2 && r == JT_OK; s++) {
        const int64_t n = b->n[s];
        if (n == 0) continue;
        const float* src = pp[s];
        if (mem == JT_MEM_HOST) {
            if (cudaMemcpyAsync(stage, src, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, B->st) != cudaSuccess)
                r = JT_ECUDA;
            src = stage;
        }
        jt_launch_aos_in(src, n, b->pos[s], b->id[s], B->st);
        if (vv[s]) {
            const float* vs = vv[s];
            if (mem == JT_MEM_HOST) {
                cudaStreamSynchronize(B->st);
                if (cudaMemcpyAsync(stage, vs, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, B->st) != cudaSuccess)
                    r = JT_ECUDA;
                vs = stage;
            }
            jt_launch_aos_in(vs, n, b->vel[s], nullptr, B->st);
        } else {
            cudaMemsetAsync(b->vel[s], 0, sizeof(float4) * n, B->st);
        }
        if (cudaStreamSynchronize(B->st) != cudaSuccess) r = JT_ECUDA;
    }
    if (r == JT_OK && cudaGetLastError() != cudaSuccess) r = JT_ECUDA;
    if (r != JT_OK) {
        jt_batch_remove(B, id);
        return r;
    }
    *box_id = id;
    return JT_OK;
}

int jt_batch_prepare(jt_batch* B, int pm_grid)
{
    if (!B || pm_grid < 8 || pm_grid > 1024 || (pm_grid & (pm_grid - 1))) return JT_EINVAL;
    AllocScope scope(&B->actx);
    Bucket& k = B->buckets[pm_grid];
    k.M = pm_grid;
    if (!k.decided) {
        k.fused = zfft_for(pm_grid);
        k.decided = true;
    }
    // every batch an execution can take: the powers of two up to the chunk
    const int ch = fft_chunk(pm_grid);
    for (int b = 1; b <= ch; b <<= 1) {
        JT_TRY(make_plan(B, k.r2c, pm_grid, b, true, k.fused));
        JT_TRY(make_plan(B, k.c2r, pm_grid, b, false, k.fused));
    }
    return JT_OK;
}

int jt_batch_set_screening(jt_batch* B, int box_id, double lambda_0, double z)
{
    if (!box_id_ok(B, box_id) || !(lambda_0 >= 0.0) || !(z > -1.0) || !std::isfinite(lambda_0) ||
        !std::isfinite(z))
        return JT_EINVAL;
    AllocScope scope(&B->actx);
    jt_box_state* b = B->boxes[box_id];
    const double kappa = lambda_0 > 0.01 ? 1.0 / (lambda_0 * std::sqrt(1.0 + z)) : 0.0;
    if (kappa == b->kappa && (kappa == 0.0) == (b->ytab == nullptr)) return JT_OK;
    const size_t ntab = (size_t)JT_LTAB_N;
    if (kappa == 0.0) {
        dfree(b->ytab);
        b->bytes -= sizeof(float2) * ntab;
    } else {
        std::vector<float2> tab(ntab);
        jt_yukawa_log_table(kappa * b->cfg.r_s, tab.data());
        if (!b->ytab) {
            JT_TRY(dalloc(&b->ytab, ntab));
            b->bytes += sizeof(float2) * ntab;
        }
        JT_CU(cudaMemcpyAsync(b->ytab, tab.data(), sizeof(float2) * ntab, cudaMemcpyHostToDevice, B->st));
        JT_CU(cudaStreamSynchronize(B->st));
    }
    b->kappa = kappa;
    b->acc_valid = false;
    B->gen++;   // the pass's kernels and grid layout change
    return JT_OK;
}

int jt_batch_remove(jt_batch* B, int box_id)
{
    if (!box_id_ok(B, box_id)) return JT_EINVAL;
    AllocScope scope(&B->actx);
    cudaStreamSynchronize(B->st);
    box_release(B->boxes[box_id]);
    B->gen++;
    delete B->boxes[box_id];
    B->boxes[box_id] = nullptr;
    return JT_OK;
}

int jt_batch_forces(jt_batch* B, const int* ids, int n_ids, int part)
{
    if (!B || part < 1 || part > 3) return JT_EINVAL;
    AllocScope scope(&B->actx);
    B->tm = jt_timings{};
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaEventRecord(t0, B->st);
    int r = jtb_force_pass(B, ids, n_ids, part, 0.0f, nullptr);
    cudaEventRecord(t1, B->st);
    int e = finish(B);
    if (r == JT_OK) r = e;
    if (r == JT_OK) B->tm.total_ms = elapsed(t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    return r;
}

int jt_batch_step(jt_batch* B, const int* ids, int n_ids, const jt_step_args* args, int nsteps)
{
    if (!B || nsteps < 0 || !args) return JT_EINVAL;
    AllocScope scope(&B->actx);
    std::vector<int> v;
    JT_TRY(valid_ids(B, ids, n_ids, v));
    std::vector<jt_box_step> steps(v.size());
    for (size_t k = 0; k < v.size(); k++) {
        const jt_step_args& a = args[k];
        if (!std::isfinite(a.dt) || !std::isfinite(a.hubble) || !std::isfinite(a.dtau_per_dt)) return JT_EINVAL;
        // FP64 step factors, applied in FP32 (kicks and drifts use 0.5 dt and
        // dt; halving a float is exact)
        steps[k].dt = (float)a.dt;
        steps[k].drag = (float)(a.hubble * a.dtau_per_dt);
    }
    if (nsteps == 0) return JT_OK;
    B->tm = jt_timings{};
    cudaEvent_t t0, t1, k0, k1;
    cudaEventCreate(&t0); cudaEventCreate(&t1); cudaEventCreate(&k0); cudaEventCreate(&k1);
    cudaEventRecord(t0, B->st);
    int r = JT_OK;
    // the opening half kick needs forces at the current positions: compute
    // them for the boxes that lack them (new or restored boxes), not for the
    // whole set
    std::vector<int> need;
    std::vector<jt_box_step> need_steps;
    for (size_t k = 0; k < v.size(); k++)
        if (!B->boxes[v[k]]->acc_valid) {
            need.push_back(v[k]);
            need_steps.push_back(steps[k]);
        }
    // its completion is awaited after the next plan is built, so that the
    // host's plan work for the step overlaps the pass on the device (the
    // new plan's tables reach the device in stream order, after the pass)
    bool open_pending = false;
    if (!need.empty()) {
        r = jtb_force_pass(B, need.data(), (int)need.size(), JT_PART_ALL, 0.0f, need_steps.data());
        open_pending = r == JT_OK;
    }
    double kd = 0.0;
    if (open_pending && B->use_graphs) {
        r = finish(B);
        open_pending = false;
    }
    if (r == JT_OK && B->use_graphs) {
        if (B->gc.gen != B->gen || B->gc.ids != v) r = capture_graphs(B, v, steps.data());
        if (r == JT_OK) {
            // this call's dt and drag into the graphs' box table
            Plan& G = B->gc.plan;
            for (size_t k = 0; k < v.size(); k++) {
                G.bx[k].dt = steps[k].dt;
                G.bx[k].kick_drag = steps[k].drag;
            }
            r = cudaMemcpyAsync((void*)G.d_bx, G.bx.data(), sizeof(jt_box_dev) * G.bx.size(),
                                cudaMemcpyHostToDevice, B->st) == cudaSuccess ? JT_OK : JT_ECUDA;
        }
        for (int k = 0; k < nsteps && r == JT_OK; k++) {
            const int parity = B->boxes[B->gc.box0]->pos[B->gc.sp0] == B->gc.pre0 ? 0 : 1;
            if (cudaGraphLaunch(B->gc.exec[parity], B->st) != cudaSuccess) {
                r = JT_ECUDA;
                break;
            }
            swap_state(B, v);
            for (int id : v) B->boxes[id]->acc_valid = true;
            B->tm.launches += B->gc.launches;
        }
        if (r == JT_OK) r = finish(B);
        nsteps = 0;   // all steps ran as graphs
    }
    Plan& P = B->plan;
    if (r == JT_OK && nsteps > 0) r = build_plan(B, v, steps.data(), P);
    if (open_pending) {
        const int rf = finish(B);
        if (r == JT_OK) r = rf;
    }
    for (int k = 0; k < nsteps && r == JT_OK; k++) {
        cudaEventRecord(k0, B->st);
        if (k == 0) jt_b_kick_drift(P.d_pre, P.d_bx, P.d_pp, (int)P.pre.size(), P.npart, 0.5f, 1.0f, B->st);
        else jt_b_drift(P.d_pre, P.d_bx, P.d_pp, (int)P.pre.size(), P.npart, 1.0f, B->st);
        B->tm.launches += 1;
        cudaEventRecord(k1, B->st);
        // closing half kick, merged with the next step's opening half kick
        r = force_pass(B, P, JT_PART_ALL, k + 1 < nsteps ? 1.0f : 0.5f);
        if (r != JT_OK) break;
        r = finish(B);
        if (r != JT_OK) break;
        kd += elapsed(k0, k1);
    }
    cudaEventRecord(t1, B->st);
    if (cudaStreamSynchronize(B->st) != cudaSuccess && r == JT_OK) r = JT_ECUDA;
    if (r == JT_OK) {
        B->tm.total_ms = elapsed(t0, t1);
        B->tm.kick_drift_ms = kd;
    }
    cudaEventDestroy(t0); cudaEventDestroy(t1); cudaEventDestroy(k0); cudaEventDestroy(k1);
    return r;
}

int jt_batch_get_accel(jt_batch* B, int box_id, float* acc_p, float* acc_m, int mem)
{
    if (!box_id_ok(B, box_id) || (mem != JT_MEM_HOST && mem != JT_MEM_DEVICE)) return JT_EINVAL;
    AllocScope scope(&B->actx);
    jt_box_state* b = B->boxes[box_id];
    if (!b->acc_valid) return JT_ESTATE;
    JT_TRY(read_out(B, b->acc[0], b->id[0], b->n[0], acc_p, mem));
    JT_TRY(read_out(B, b->acc[1], b->id[1], b->n[1], acc_m, mem));
    JT_CU(cudaStreamSynchronize(B->st));
    return JT_OK;
}

int jt_batch_get_state(jt_batch* B, int box_id, float* pos_p, float* vel_p, float* pos_m, float* vel_m, int mem)
{
    if (!box_id_ok(B, box_id) || (mem != JT_MEM_HOST && mem != JT_MEM_DEVICE)) return JT_EINVAL;
    AllocScope scope(&B->actx);
    jt_box_state* b = B->boxes[box_id];
    JT_TRY(read_out(B, b->pos[0], b->id[0], b->n[0], pos_p, mem));
    JT_TRY(read_out(B, b->vel[0], b->id[0], b->n[0], vel_p, mem));
    JT_TRY(read_out(B, b->pos[1], b->id[1], b->n[1], pos_m, mem));
    JT_TRY(read_out(B, b->vel[1], b->id[1], b->n[1], vel_m, mem));
    JT_CU(cudaStreamSynchronize(B->st));
    return JT_OK;
}

int jt_batch_box_info(jt_batch* B, int box_id, size_t* n_p, size_t* n_m, size_t* bytes)
{
    if (!box_id_ok(B, box_id)) return JT_EINVAL;
    jt_box_state* b = B->boxes[box_id];
    if (n_p) *n_p = (size_t)b->n[0];
    if (n_m) *n_m = (size_t)b->n[1];
    if (bytes) *bytes = b->bytes;
    return JT_OK;
}

int jt_batch_memory(jt_batch* B, size_t* persistent, size_t* scratch)
{
    if (!B) return JT_EINVAL;
    size_t p = 0, s = 0;
    for (auto* b : B->boxes)
        if (b) p += b->bytes;
    s += B->child.bytes() + B->range.bytes() + B->parent.bytes() + B->flag.bytes() + B->com.bytes() +
         B->bmin.bytes() + B->bmax.bytes() + B->quad0.bytes() + B->quad1.bytes() + B->m30.bytes() +
         B->vals.bytes() + B->vals_alt.bytes() + B->keys_alt.bytes() + B->hist.bytes() + B->status.bytes() +
         B->tickets.bytes() + B->desc.bytes() + B->fftws.bytes() + B->gdesc.bytes() + B->stage.bytes();
    for (auto& kv : B->buckets) s += (size_t)kv.second.cap * grid_bytes(kv.first, B->ngrid);
    if (persistent) *persistent = p;
    if (scratch) *scratch = s;
    return JT_OK;
}

int jt_batch_estimate(const jt_config* cfg, size_t n_p, size_t n_m, size_t* persistent, size_t* scratch)
{
    if (validate_box_config(cfg) != JT_OK) return JT_EINVAL;
    const size_t n = n_p + n_m;
    const int64_t M = cfg->pm_grid;
    if (persistent) *persistent = n * (5 * sizeof(float4) + 2 * sizeof(int)) + 2 * (size_t)M * sizeof(float4);
    if (scratch) {
        // tree: 2n nodes (child, parent, com, bmin, bmax, quad0, quad1) and n
        // (range, flag); sort: m30, vals, vals_alt, keys_alt and the look-back
        // words (4 passes x 256 per 4096-element tile); PM grids of one box
        size_t tree = 2 * n * (sizeof(int2) + sizeof(int) + 4 * sizeof(float4) + sizeof(float2)) +
                      n * (sizeof(int2) + sizeof(int));
        size_t sort = n * 4 * sizeof(uint32_t) + (n / 4096 + 2) * 4 * 256 * sizeof(uint32_t);
        // near-field cell list (cpos, cid, ccell, cslot, tflag per particle)
        // and the interpolated PM accelerations (one float4 per grid)
        size_t cells = n * (sizeof(float4) + sizeof(int2) + 2 * sizeof(int) + 1) +
                       n * box_ngrid(*cfg) * sizeof(float4);
        *scratch = tree + sort + cells + grid_bytes(M, box_ngrid(*cfg));
    }
    return JT_OK;
}

int jt_batch_set_graphs(jt_batch* B, int on)
{
    if (!B) return JT_EINVAL;
    B->use_graphs = on != 0;
    if (!on) drop_graphs(B);
    return JT_OK;
}

int jt_batch_set_counters(jt_batch* B, int on)
{
    if (!B) return JT_EINVAL;
    if (B->counters != (on != 0)) drop_graphs(B);   // the graphs hold the walk's variant
    B->counters = on != 0;
    return JT_OK;
}

int jt_batch_trim(jt_batch* B)
{
    if (!B) return JT_EINVAL;
    AllocScope scope(&B->actx);
    if (cudaStreamSynchronize(B->st) != cudaSuccess) return JT_ECUDA;
    drop_graphs(B);
    B->child.release(); B->range.release(); B->parent.release(); B->flag.release();
    B->com.release(); B->bmin.release(); B->bmax.release(); B->quad0.release(); B->quad1.release();
    B->ccount.release(); B->cstart.release(); B->cbsum.release(); B->ccell.release(); B->cslot.release();
    B->csegflag.release();
    B->cpos.release(); B->cid.release(); B->tflag.release(); B->pmacc.release();
    B->m30.release(); B->vals.release(); B->vals_alt.release(); B->keys_alt.release();
    B->hist.release(); B->status.release(); B->tickets.release();
    for (auto& kv : B->buckets) kv.second.release();
    B->buckets.clear();
    B->fftws.release();
    B->fft_need = 0;
    B->fft_dirty = false;
    B->stage.release();
    B->gen++;
    // hand the freed blocks back to the device
    if (cudaStreamSynchronize(B->st) != cudaSuccess) return JT_ECUDA;
    cudaMemPoolTrimTo(B->actx.pool, 0);
    return JT_OK;
}

int jt_batch_get_timings(jt_batch* B, jt_timings* t)
{
    if (!B || !t) return JT_EINVAL;
    *t = B->tm;
    return JT_OK;
}

}  // extern "C"

int jtb_reserve(jt_batch* B, size_t bytes)
{
    if (!B) return JT_EINVAL;
    if (bytes == 0) return JT_OK;
    void* p = nullptr;
    if (cudaMallocFromPoolAsync(&p, bytes, B->actx.pool, B->st) != cudaSuccess) {
        cudaGetLastError();
        return JT_ENOMEM;
    }
    JT_CU(cudaFreeAsync(p, B->st));
    JT_CU(cudaStreamSynchronize(B->st));
    return JT_OK;
}

std::string jt_cell_tuning_text()
{
    std::lock_guard<std::mutex> lock(g_cell_tune_mu);
    return g_cell_tune_text;
}

void jtb_set_cell_tune(jt_batch* B, bool on)
{
    if (B) B->cell_tune = on;
}
