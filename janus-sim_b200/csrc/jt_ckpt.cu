// Checkpoints that overlap the next step, and the production driver's raw
// snapshot format.
//
// jt_batch_checkpoint_async: the box's state is gathered into caller order
// in a device scratch on the batch's stream (one kernel per array), an event
// marks the gather, a side stream copies the scratch to pinned host memory
// after that event, and a host thread waits for the copy and writes the
// snapshot_v3 file (jt_snapshot_write).  The call returns as soon as the
// work is enqueued: the next jt_batch_step on the batch's stream overlaps the
// copy and the file write (the scratch is touched by nothing else until the
// checkpoint is collected).  One checkpoint per batch is in flight;
// jt_batch_checkpoint_wait collects it.  The reference writes its snapshots
// synchronously after a blocking device-to-host copy of every particle
// (src/snapshot_v3.rs:260-376, src/bin/janus_mu19_production.rs:198-216).
//
// Raw format (save_snapshot, src/bin/janus_mu19_production.rs:198-216): u32
// n, f32 box, u32 step, f32 z, then n records of f32 pos[3], f32 vel[3], i8
// sign (25 bytes, little-endian, no padding).
#include "jt_batch.h"

#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

struct jt_ckpt {
    int device = 0;
    cudaStream_t side = nullptr;
    cudaEvent_t gathered = nullptr, copied = nullptr;
    float* dev = nullptr;
    size_t dev_cap = 0;          // floats
    float* host = nullptr;       // pinned
    size_t host_cap = 0;         // floats
    std::thread worker;
    bool active = false;
    int result = JT_OK;
};

namespace {

int ensure(jt_ckpt* c, size_t floats)
{
    if (c->dev_cap < floats) {
        if (c->dev) cudaFree(c->dev);
        c->dev = nullptr;
        c->dev_cap = 0;
        if (cudaMalloc(&c->dev, sizeof(float) * floats) != cudaSuccess) {
            cudaGetLastError();
            return JT_ENOMEM;
        }
        c->dev_cap = floats;
    }
    if (c->host_cap < floats) {
        if (c->host) cudaFreeHost(c->host);
        c->host = nullptr;
        c->host_cap = 0;
        if (cudaMallocHost(&c->host, sizeof(float) * floats) != cudaSuccess) {
            cudaGetLastError();
            return JT_ENOMEM;
        }
        c->host_cap = floats;
    }
    return JT_OK;
}

void join(jt_ckpt* c)
{
    if (c && c->worker.joinable()) c->worker.join();
}

template <class T>
void put(std::vector<unsigned char>& b, T v)
{
    unsigned char t[sizeof(T)];
    std::memcpy(t, &v, sizeof(T));
    b.insert(b.end(), t, t + sizeof(T));
}

}  // namespace

void jt_ckpt_release(jt_ckpt* c)
{
    if (!c) return;
    join(c);
    if (c->side) cudaStreamSynchronize(c->side);
    if (c->gathered) cudaEventDestroy(c->gathered);
    if (c->copied) cudaEventDestroy(c->copied);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->dev) cudaFree(c->dev);
    if (c->host) cudaFreeHost(c->host);
    delete c;
}

extern "C" {

int jt_batch_checkpoint_async(jt_batch* B, int box_id, const char* path, const jt_snapshot_meta* meta)
{
    jt_box_state* b = jtb_box(B, box_id);
    if (!b || !path || !meta) return JT_EINVAL;
    jt_ckpt** slot = jtb_ckpt_slot(B);
    if (!*slot) {
        jt_ckpt* c = new jt_ckpt();
        cudaGetDevice(&c->device);
        if (cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&c->gathered, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&c->copied, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            jt_ckpt_release(c);
            return JT_ECUDA;
        }
        *slot = c;
    }
    jt_ckpt* c = *slot;
    join(c);   // one checkpoint in flight; the previous one's result is kept until collected
    if (c->active) return JT_EBUSY;
    const int64_t np = b->n[0], nm = b->n[1], n = np + nm;
    if (n == 0) return JT_ESTATE;
    int r = ensure(c, 6 * (size_t)n);
    if (r != JT_OK) return r;
    cudaStream_t st = jtb_stream(B);
    // caller order: [pos_p, pos_m] then [vel_p, vel_m], AoS float3
    float* pos = c->dev;
    float* vel = c->dev + 3 * n;
    if (np) {
        jt_launch_aos_out(b->pos[0], b->id[0], nullptr, np, pos, st);
        jt_launch_aos_out(b->vel[0], b->id[0], nullptr, np, vel, st);
    }
    if (nm) {
        jt_launch_aos_out(b->pos[1], b->id[1], nullptr, nm, pos + 3 * np, st);
        jt_launch_aos_out(b->vel[1], b->id[1], nullptr, nm, vel + 3 * np, st);
    }
    if (cudaGetLastError() != cudaSuccess || cudaEventRecord(c->gathered, st) != cudaSuccess ||
        cudaStreamWaitEvent(c->side, c->gathered, 0) != cudaSuccess ||
        cudaMemcpyAsync(c->host, c->dev, sizeof(float) * 6 * n, cudaMemcpyDeviceToHost, c->side) != cudaSuccess ||
        cudaEventRecord(c->copied, c->side) != cudaSuccess)
        return JT_ECUDA;
    const std::string file(path);
    const jt_snapshot_meta m = *meta;
    const double L = b->cfg.box_L, mu = b->cfg.mu, eps = b->cfg.softening;
    const float mp = b->mass[0], mm = b->mass[1];
    c->active = true;
    c->result = JT_OK;
    c->worker = std::thread([c, file, m, L, mu, eps, mp, mm, np, nm]() {
        cudaSetDevice(c->device);
        if (cudaEventSynchronize(c->copied) != cudaSuccess) {
            c->result = JT_ECUDA;
            return;
        }
        const int64_t n = np + nm;
        std::vector<int8_t> sg(n);
        std::vector<float> mass(n), ep(n, (float)eps);
        for (int64_t i = 0; i < n; i++) {
            sg[i] = i < np ? 1 : -1;
            mass[i] = i < np ? mp : mm;
        }
        c->result = jt_snapshot_write(file.c_str(), &m, L, mu, c->host, c->host + 3 * n, sg.data(), mass.data(),
                                      ep.data(), (size_t)n);
    });
    return JT_OK;
}

int jt_batch_checkpoint_wait(jt_batch* B)
{
    if (!B) return JT_EINVAL;
    jt_ckpt* c = *jtb_ckpt_slot(B);
    if (!c || !c->active) return JT_OK;
    join(c);
    c->active = false;
    return c->result;
}

int jt_snapshot_write_raw(const char* path, const float* pos, const float* vel, const int8_t* signs, size_t n,
                          double box_L, uint32_t step, double z)
{
    if (!path || (n && (!pos || !signs)) || n > 0xFFFFFFFFull) return JT_EINVAL;
    std::vector<unsigned char> b;
    b.reserve(16 + 25 * n);
    put<uint32_t>(b, (uint32_t)n);
    put<float>(b, (float)box_L);
    put<uint32_t>(b, step);
    put<float>(b, (float)z);
    for (size_t i = 0; i < n; i++) {
        for (int d = 0; d < 3; d++) put<float>(b, pos[3 * i + d]);
        for (int d = 0; d < 3; d++) put<float>(b, vel ? vel[3 * i + d] : 0.0f);
        put<int8_t>(b, signs[i]);
    }
    FILE* f = std::fopen(path, "wb");
    if (!f) return JT_EINVAL;
    const bool ok = std::fwrite(b.data(), 1, b.size(), f) == b.size();
    return (std::fclose(f) == 0 && ok) ? JT_OK : JT_EINVAL;
}

int jt_snapshot_read_raw(const char* path, float* pos, float* vel, int8_t* signs, size_t cap, size_t* n,
                         double* box_L, uint32_t* step, double* z)
{
    if (!path || !n) return JT_EINVAL;
    FILE* f = std::fopen(path, "rb");
    if (!f) return JT_EINVAL;
    unsigned char h[16];
    if (std::fread(h, 1, 16, f) != 16) {
        std::fclose(f);
        return JT_EINVAL;
    }
    uint32_t nn, st;
    float L, zz;
    std::memcpy(&nn, h, 4);
    std::memcpy(&L, h + 4, 4);
    std::memcpy(&st, h + 8, 4);
    std::memcpy(&zz, h + 12, 4);
    *n = nn;
    if (box_L) *box_L = L;
    if (step) *step = st;
    if (z) *z = zz;
    if (!pos) {
        std::fclose(f);
        return JT_OK;
    }
    if (cap < nn || !signs) {
        std::fclose(f);
        return JT_EINVAL;
    }
    std::vector<unsigned char> rec((size_t)25 * nn);
    const bool ok = std::fread(rec.data(), 1, rec.size(), f) == rec.size();
    std::fclose(f);
    if (!ok) return JT_EINVAL;
    for (size_t i = 0; i < nn; i++) {
        const unsigned char* q = rec.data() + 25 * i;
        std::memcpy(pos + 3 * i, q, 12);
        if (vel) std::memcpy(vel + 3 * i, q + 12, 12);
        std::memcpy(signs + i, q + 24, 1);
    }
    return JT_OK;
}

}  // extern "C"
