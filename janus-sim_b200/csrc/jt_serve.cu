// Serving loop: simulation jobs admitted by an HBM budget, continuous
// batching of their step requests, eviction to pinned host memory.
//
// The reference has no server: its parameter scans launch one process per
// box (optim/run_tour.py:40-48) and each process owns the whole GPU.  Here a
// jt_server owns one jt_batch and a set of jobs:
//   * a job is one box (config + state in pinned host memory + the number of
//     steps it wants);
//   * step requests arrive over time (jt_server_request, or a timed arrival
//     schedule replayed in real time by jt_server_serve); each job keeps a
//     FIFO of pending requests;
//   * admission: a queued job with a pending request is moved to the device
//     (jt_batch_add) when its persistent state plus the per-pass scratch of
//     every resident job (jt_batch_estimate) still fits the HBM budget,
//     first come first served by the job's oldest request; a job that does
//     not fit first swaps idle resident jobs (no pending request) out to
//     their pinned host buffers, least recently served first;
//   * continuous batching: each batched step advances EVERY resident job
//     that has a pending request by one KDK step, in one launch per stage;
//     requests that arrive while a step runs join the next one;
//   * completion: a job that has taken all its steps is evicted: its state is
//     copied into its pinned host buffers and its device memory freed.
// Latency of a request = end of the batched step that served it minus its
// arrival time (host clock), including any wait for admission.
#include "jt_batch.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <new>
#include <set>
#include <thread>
#include <vector>

namespace {

enum JobState { kQueued = JT_JOB_QUEUED, kResident = JT_JOB_RESIDENT, kDone = JT_JOB_DONE };

struct Job {
    jt_config cfg;
    size_t n_p = 0, n_m = 0;
    float* host = nullptr;         // pinned: pos_p, vel_p, pos_m, vel_m (3 floats each)
    float* host_acc = nullptr;     // pinned: acc_p, acc_m of a swapped-out job
    float* dev_host = nullptr;     // device addresses of the same pinned buffers
    float* dev_host_acc = nullptr;
    bool acc_saved = false;        // host_acc belongs to the state in host
    int steps_total = 0, steps_done = 0;
    jt_step_args args = {0.0, 0.0, 1.0};
    int state = kQueued;
    int box = -1;
    size_t persistent = 0, scratch = 0;
    size_t fft_ws = 0;             // cuFFT work area its grids may need
    std::deque<double> pending;    // arrival times of outstanding step requests
    double last_served = -1.0;     // server clock of the last step it took
};

double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

}  // namespace

struct jt_server {
    jt_batch* B = nullptr;
    size_t budget = 0;
    size_t resident_persistent = 0, resident_scratch = 0;
    std::vector<Job> jobs;
    std::vector<double> lat;       // per served request, seconds
    double t0 = 0.0;               // clock origin of arrival times
    int64_t steps = 0, particle_steps = 0, admitted = 0, evicted = 0, refused_fit = 0, swapped = 0;
    int64_t trims = 0;
    double busy_s = 0.0;
    size_t peak_device = 0;
    double admit_s = 0.0, evict_s = 0.0;   // wall time in admissions / evictions
    double step_device_s = 0.0;            // device time of the batched steps
    jt_timings tm_sum{};                   // their stage times and counts, summed
    size_t reserved = 0;                   // bytes reserved in the batch's pool at creation
    int max_resident = 0;
    std::set<int> prepared;        // grid sizes whose cuFFT plans the batch holds (jt_batch_prepare)
};

namespace {

size_t device_bytes(jt_server* S)
{
    size_t p = 0, s = 0;
    jt_batch_memory(S->B, &p, &s);
    return p + s;
}

int admit(jt_server* S, Job& j)
{
    const double t_in = now_s();
    struct Clock {
        jt_server* S;
        double t;
        ~Clock() { S->admit_s += now_s() - t; }
    } clock_{S, t_in};
    const float* h = j.dev_host;
    const size_t np = j.n_p, nm = j.n_m;
    int box = -1;
    int r = jtb_add_empty(S->B, &j.cfg, (int64_t)np, (int64_t)nm, &box);
    if (r != JT_OK) return r;
    // the state (and, for a swapped-out job, its forces: no extra force pass)
    // read from the job's pinned buffers by kernels queued on the batch's
    // stream, without a host wait: the next step runs after them in stream order
    const float* pos[2] = {h, h + 6 * np};
    const float* vel[2] = {h + 3 * np, h + 6 * np + 3 * nm};
    const float* acc[2] = {j.dev_host_acc, j.dev_host_acc + 3 * np};
    r = jtb_upload_async(S->B, box, pos, vel, j.acc_saved ? acc : nullptr);
    if (r != JT_OK) {
        jt_batch_remove(S->B, box);
        return r;
    }
    j.box = box;
    j.state = kResident;
    S->resident_persistent += j.persistent;
    S->resident_scratch += j.scratch;
    S->admitted++;
    return JT_OK;
}

// Copy a resident job's state to its pinned host buffers and free its device
// memory; final = the job has taken all its steps (else it is swapped out
// and re-admitted when it has a request again).
int evict(jt_server* S, Job& j, bool final)
{
    struct Clock {
        jt_server* S;
        double t;
        ~Clock() { S->evict_s += now_s() - t; }
    } clock_{S, now_s()};
    float* h = j.dev_host;
    const size_t np = j.n_p, nm = j.n_m;
    // the state and the forces at it (none yet: a swapped-out job then comes
    // back with a force pass; a finished job's forces are its result as much
    // as its state, jt_server_get_accel) into the job's pinned buffers, and
    // the box's memory freed, all in the batch's stream order with no host
    // wait; readers of the buffers synchronise the stream first
    float* pos[2] = {h, h + 6 * np};
    float* vel[2] = {h + 3 * np, h + 6 * np + 3 * nm};
    float* acc[2] = {j.dev_host_acc, j.dev_host_acc + 3 * np};
    bool got_acc = false;
    int r = jtb_download_async(S->B, j.box, pos, vel, acc, &got_acc);
    if (r != JT_OK) return r;
    j.acc_saved = got_acc;
    r = jtb_remove_async(S->B, j.box);
    if (r != JT_OK) return r;
    j.box = -1;
    j.state = final ? kDone : kQueued;
    S->resident_persistent -= j.persistent;
    S->resident_scratch -= j.scratch;
    if (final) S->evicted++;
    else S->swapped++;
    return JT_OK;
}

// cuFFT work area a job's transforms may need: one execution covers at most
// 2^27 real elements (jt_batch.cu), so at most 2^27 complex elements.
size_t fft_ws_of(const jt_config& c)
{
    const size_t G = (size_t)c.pm_grid * c.pm_grid * c.pm_grid;
    return 8 * std::min((size_t)6 * G, (size_t)1 << 27);
}

// Device bytes of a set of jobs: persistent state, per-pass scratch with the
// pools' 1/16 growth headroom, and the batch's shared cuFFT work area (the
// largest any of them needs).
size_t need_of(size_t persistent, size_t scratch, size_t fft_ws)
{
    return persistent + scratch + scratch / 16 + fft_ws;
}

int trim(jt_server* S)
{
    S->trims++;
    S->prepared.clear();   // the trim releases the plans too
    int r = jt_batch_trim(S->B);
    // map the reservation again (the trim returned it to the device)
    if (r == JT_OK && S->reserved) jtb_reserve(S->B, S->reserved);
    return r;
}

bool fits(jt_server* S, const Job& j)
{
    size_t ws = j.fft_ws;
    for (const Job& q : S->jobs)
        if (q.state == kResident) ws = std::max(ws, q.fft_ws);
    return need_of(S->resident_persistent + j.persistent, S->resident_scratch + j.scratch, ws) <= S->budget;
}

int admit_waiting(jt_server* S)
{
    std::vector<int> order;
    for (size_t k = 0; k < S->jobs.size(); k++)
        if (S->jobs[k].state == kQueued && !S->jobs[k].pending.empty()) order.push_back((int)k);
    std::sort(order.begin(), order.end(),
              [&](int a, int b) { return S->jobs[a].pending.front() < S->jobs[b].pending.front(); });
    for (int k : order) {
        Job& j = S->jobs[k];
        if (!fits(S, j)) {
            std::vector<int> idle;
            for (size_t q = 0; q < S->jobs.size(); q++)
                if (S->jobs[q].state == kResident && S->jobs[q].pending.empty()) idle.push_back((int)q);
            std::sort(idle.begin(), idle.end(),
                      [&](int a, int b) { return S->jobs[a].last_served < S->jobs[b].last_served; });
            for (int q : idle) {
                if (fits(S, j)) break;
                int r = evict(S, S->jobs[q], false);
                if (r != JT_OK) return r;
            }
        }
        if (!fits(S, j)) {
            S->refused_fit++;
            break;      // first come, first served: later jobs wait behind it
        }
        // the batch's scratch pools only grow: release them when what they
        // hold plus this job would pass the budget (they regrow to what the
        // resident jobs need)
        size_t pers = 0, scr = 0;
        jt_batch_memory(S->B, &pers, &scr);
        if (pers + j.persistent + std::max(scr, S->resident_scratch + j.scratch) > S->budget) {
            int r = trim(S);
            if (r != JT_OK) return r;
        }
        int r = admit(S, j);
        if (r == JT_ENOMEM) {
            // scratch pools held for an earlier mix: release them and retry
            r = trim(S);
            if (r == JT_OK) r = admit(S, j);
        }
        if (r == JT_ENOMEM) break;     // the device disagrees with the estimate: retry later
        if (r != JT_OK) return r;
    }
    return JT_OK;
}

// One batched step of every resident job with a pending request.
int step_once(jt_server* S, int* served)
{
    *served = 0;
    std::vector<int> ids, jix;
    std::vector<jt_step_args> args;
    for (size_t k = 0; k < S->jobs.size(); k++) {
        Job& j = S->jobs[k];
        if (j.state == kResident && !j.pending.empty()) {
            ids.push_back(j.box);
            jix.push_back((int)k);
            args.push_back(j.args);
        }
    }
    if (ids.empty()) return JT_OK;
    const double a = now_s();
    int r = jt_batch_step(S->B, ids.data(), (int)ids.size(), args.data(), 1);
    if (r == JT_ENOMEM) {
        // the pass could not grow its scratch (pools sized for an earlier
        // mix of jobs, fragmentation): release every pool and retry once;
        // no kernel ran before the allocation failed
        r = trim(S);
        if (r == JT_OK) r = jt_batch_step(S->B, ids.data(), (int)ids.size(), args.data(), 1);
    }
    if (r != JT_OK) return r;
    const double done = now_s();
    S->busy_s += done - a;
    {
        jt_timings t;
        if (jt_batch_get_timings(S->B, &t) == JT_OK) {
            S->step_device_s += 1e-3 * t.total_ms;
            jt_timings& a = S->tm_sum;
            a.sort_ms += t.sort_ms;
            a.tree_ms += t.tree_ms;
            a.deposit_ms += t.deposit_ms;
            a.fft_ms += t.fft_ms;
            a.kspace_ms += t.kspace_ms;
            a.walk_ms += t.walk_ms;
            a.kick_drift_ms += t.kick_drift_ms;
            a.total_ms += t.total_ms;
            a.interactions += t.interactions;
            a.launches += t.launches;
            a.pair_interactions += t.pair_interactions;
            a.node_interactions += t.node_interactions;
            a.candidates += t.candidates;
            a.cellwalk_ms += t.cellwalk_ms;
            a.interp_ms += t.interp_ms;
        }
    }
    S->steps++;
    S->max_resident = std::max(S->max_resident, (int)ids.size());
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess)
        S->peak_device = std::max(S->peak_device, total_b - free_b);   // whole device, context included
    else
        S->peak_device = std::max(S->peak_device, device_bytes(S));
    for (int k : jix) {
        Job& j = S->jobs[k];
        S->lat.push_back(done - S->t0 - j.pending.front());
        j.pending.pop_front();
        j.steps_done++;
        j.last_served = done - S->t0;
        S->particle_steps += (int64_t)(j.n_p + j.n_m);
        if (j.steps_done >= j.steps_total) {
            r = evict(S, j, true);
            if (r != JT_OK) return r;
        }
    }
    *served = (int)jix.size();
    return JT_OK;
}

double percentile(std::vector<double> v, double q)
{
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    double pos = q * (double)(v.size() - 1);
    size_t i = (size_t)pos;
    double f = pos - (double)i;
    return i + 1 < v.size() ? v[i] * (1.0 - f) + v[i + 1] * f : v[i];
}

bool job_ok(jt_server* S, int job) { return S && job >= 0 && job < (int)S->jobs.size(); }

}  // namespace

extern "C" {

int jt_server_create(size_t hbm_budget_bytes, jt_server** out)
{
    if (!out || hbm_budget_bytes == 0) return JT_EINVAL;
    *out = nullptr;
    jt_server* S = new (std::nothrow) jt_server();
    if (!S) return JT_ENOMEM;
    int r = jt_batch_create(&S->B);
    if (r != JT_OK) {
        delete S;
        return r;
    }
    jtb_set_cell_tune(S->B, false);   // no timing runs inside a request's step
    S->budget = hbm_budget_bytes;
    // map the budget once, up front (see the header)
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
        const size_t want = std::min(hbm_budget_bytes, free_b / 10 * 9);
        if (jtb_reserve(S->B, want) == JT_OK) S->reserved = want;
    }
    S->t0 = now_s();
    *out = S;
    return JT_OK;
}

void jt_server_destroy(jt_server* S)
{
    if (!S) return;
    jt_batch_destroy(S->B);
    for (Job& j : S->jobs) {
        if (j.host) cudaFreeHost(j.host);
        if (j.host_acc) cudaFreeHost(j.host_acc);
    }
    delete S;
}

int jt_server_add_job(jt_server* S, const jt_config* cfg, const float* pos_p, const float* vel_p, size_t n_p,
                      const float* pos_m, const float* vel_m, size_t n_m, int steps_total,
                      const jt_step_args* args, int* job_id)
{
    if (!S || !cfg || !args || !job_id || steps_total <= 0 || n_p + n_m == 0) return JT_EINVAL;
    if ((n_p && !pos_p) || (n_m && !pos_m)) return JT_EINVAL;
    if (!std::isfinite(args->dt) || !std::isfinite(args->hubble) || !std::isfinite(args->dtau_per_dt))
        return JT_EINVAL;
    Job j;
    j.cfg = *cfg;
    j.n_p = n_p;
    j.n_m = n_m;
    j.steps_total = steps_total;
    j.args = *args;
    int r = jt_batch_estimate(cfg, n_p, n_m, &j.persistent, &j.scratch);
    if (r != JT_OK) return r;
    j.fft_ws = fft_ws_of(*cfg);
    if (need_of(j.persistent, j.scratch, j.fft_ws) > S->budget) return JT_EBUSY;   // can never fit
    const size_t floats = 6 * (n_p + n_m);
    // the state and, beside it, the forces a swapped-out or finished job
    // keeps: both pinned once here (page-locking costs far more than the
    // copies, so it stays out of the admissions and evictions)
    if (cudaMallocHost((void**)&j.host, sizeof(float) * floats) != cudaSuccess) return JT_ENOMEM;
    if (cudaMallocHost((void**)&j.host_acc, sizeof(float) * 3 * (n_p + n_m)) != cudaSuccess ||
        cudaHostGetDevicePointer((void**)&j.dev_host, j.host, 0) != cudaSuccess ||
        cudaHostGetDevicePointer((void**)&j.dev_host_acc, j.host_acc, 0) != cudaSuccess) {
        cudaGetLastError();
        cudaFreeHost(j.host);
        if (j.host_acc) cudaFreeHost(j.host_acc);
        j.host = nullptr;
        j.host_acc = nullptr;
        return JT_ENOMEM;
    }
    float* h = j.host;
    std::memcpy(h, pos_p, sizeof(float) * 3 * n_p);
    if (vel_p) std::memcpy(h + 3 * n_p, vel_p, sizeof(float) * 3 * n_p);
    else std::memset(h + 3 * n_p, 0, sizeof(float) * 3 * n_p);
    if (n_m) std::memcpy(h + 6 * n_p, pos_m, sizeof(float) * 3 * n_m);
    if (vel_m) std::memcpy(h + 6 * n_p + 3 * n_m, vel_m, sizeof(float) * 3 * n_m);
    else std::memset(h + 6 * n_p + 3 * n_m, 0, sizeof(float) * 3 * n_m);
    S->jobs.push_back(j);
    *job_id = (int)S->jobs.size() - 1;
    // the cuFFT plans of a new grid size, made now rather than inside the
    // first batched steps that use them (a failure leaves them to the steps)
    if (S->prepared.insert(cfg->pm_grid).second && jt_batch_prepare(S->B, cfg->pm_grid) != JT_OK) {
        S->prepared.erase(cfg->pm_grid);
        cudaGetLastError();
    }
    return JT_OK;
}

int jt_server_job_need(const jt_config* cfg, size_t n_p, size_t n_m, size_t* bytes)
{
    if (!cfg || !bytes) return JT_EINVAL;
    size_t p = 0, s = 0;
    int r = jt_batch_estimate(cfg, n_p, n_m, &p, &s);
    if (r != JT_OK) return r;
    *bytes = need_of(p, s, fft_ws_of(*cfg));
    return JT_OK;
}

int jt_server_request(jt_server* S, int job, double t_arrival)
{
    if (!job_ok(S, job)) return JT_EINVAL;
    Job& j = S->jobs[job];
    if (j.state == kDone) return JT_ESTATE;
    if ((int)j.pending.size() + j.steps_done >= j.steps_total) return JT_EINVAL;   // more than it needs
    j.pending.push_back(t_arrival < 0.0 ? now_s() - S->t0 : t_arrival);
    return JT_OK;
}

double jt_server_clock(jt_server* S) { return S ? now_s() - S->t0 : 0.0; }

int jt_server_poll(jt_server* S, int* served)
{
    if (!S || !served) return JT_EINVAL;
    *served = 0;
    int r = admit_waiting(S);
    if (r != JT_OK) return r;
    return step_once(S, served);
}

int jt_server_serve(jt_server* S, const double* t, const int* job, int n)
{
    if (!S || n < 0 || (n > 0 && (!t || !job))) return JT_EINVAL;
    for (int k = 0; k < n; k++)
        if (!job_ok(S, job[k]) || !(t[k] >= 0.0) || (k > 0 && t[k] < t[k - 1])) return JT_EINVAL;
    S->t0 = now_s();
    int next = 0;
    int64_t outstanding = 0;
    for (;;) {
        const double now = now_s() - S->t0;
        while (next < n && t[next] <= now) {
            Job& j = S->jobs[job[next]];
            if (j.state != kDone && (int)j.pending.size() + j.steps_done < j.steps_total) {
                j.pending.push_back(t[next]);
                outstanding++;
            }
            next++;
        }
        int served = 0;
        int r = jt_server_poll(S, &served);
        if (r != JT_OK) return r;
        outstanding -= served;
        if (next >= n && outstanding <= 0) break;
        if (served == 0) {
            if (next >= n) return JT_EBUSY;    // nothing runs, nothing arrives: unservable
            const double wait = t[next] - (now_s() - S->t0);
            if (wait > 0) std::this_thread::sleep_for(std::chrono::duration<double>(std::min(wait, 0.05)));
        }
    }
    return JT_OK;
}

int jt_server_job_state(jt_server* S, int job, int* state, int* steps_done)
{
    if (!job_ok(S, job)) return JT_EINVAL;
    if (state) *state = S->jobs[job].state;
    if (steps_done) *steps_done = S->jobs[job].steps_done;
    return JT_OK;
}

int jt_server_get_state(jt_server* S, int job, float* pos_p, float* vel_p, float* pos_m, float* vel_m)
{
    if (!job_ok(S, job)) return JT_EINVAL;
    Job& j = S->jobs[job];
    if (j.state == kResident) return jt_batch_get_state(S->B, j.box, pos_p, vel_p, pos_m, vel_m, JT_MEM_HOST);
    // an eviction's copies into the pinned buffers may still be in flight
    if (cudaStreamSynchronize(jtb_stream(S->B)) != cudaSuccess) return JT_ECUDA;
    const float* h = j.host;
    const size_t np = j.n_p, nm = j.n_m;
    if (pos_p) std::memcpy(pos_p, h, sizeof(float) * 3 * np);
    if (vel_p) std::memcpy(vel_p, h + 3 * np, sizeof(float) * 3 * np);
    if (pos_m) std::memcpy(pos_m, h + 6 * np, sizeof(float) * 3 * nm);
    if (vel_m) std::memcpy(vel_m, h + 6 * np + 3 * nm, sizeof(float) * 3 * nm);
    return JT_OK;
}

int jt_server_get_accel(jt_server* S, int job, float* acc_p, float* acc_m)
{
    if (!job_ok(S, job)) return JT_EINVAL;
    Job& j = S->jobs[job];
    if (j.state == kResident) return jt_batch_get_accel(S->B, j.box, acc_p, acc_m, JT_MEM_HOST);
    if (!j.acc_saved) return JT_ESTATE;
    if (cudaStreamSynchronize(jtb_stream(S->B)) != cudaSuccess) return JT_ECUDA;
    if (acc_p) std::memcpy(acc_p, j.host_acc, sizeof(float) * 3 * j.n_p);
    if (acc_m) std::memcpy(acc_m, j.host_acc + 3 * j.n_p, sizeof(float) * 3 * j.n_m);
    return JT_OK;
}

int jt_server_set_counters(jt_server* S, int on)
{
    if (!S) return JT_EINVAL;
    return jt_batch_set_counters(S->B, on);
}

int jt_server_get_timings(jt_server* S, jt_timings* out)
{
    if (!S || !out) return JT_EINVAL;
    *out = S->tm_sum;
    return JT_OK;
}

int jt_server_stats(jt_server* S, jt_serve_stats* out)
{
    if (!S || !out) return JT_EINVAL;
    jt_serve_stats s;
    std::memset(&s, 0, sizeof(s));
    s.requests_served = (int64_t)S->lat.size();
    s.batched_steps = S->steps;
    s.particle_steps = S->particle_steps;
    s.admitted = S->admitted;
    s.evicted = S->evicted;
    s.admission_waits = S->refused_fit;
    s.p50_latency_s = percentile(S->lat, 0.50);
    s.p99_latency_s = percentile(S->lat, 0.99);
    s.max_latency_s = S->lat.empty() ? 0.0 : *std::max_element(S->lat.begin(), S->lat.end());
    s.busy_s = S->busy_s;
    s.peak_device_bytes = (int64_t)S->peak_device;
    s.admit_s = S->admit_s;
    s.evict_s = S->evict_s;
    s.max_jobs_per_step = S->max_resident;
    s.swapped_out = S->swapped;
    s.trims = S->trims;
    s.step_device_s = S->step_device_s;
    s.reserved_gb = 1e-9 * (double)S->reserved;
    *out = s;
    return JT_OK;
}

}  // extern "C"
