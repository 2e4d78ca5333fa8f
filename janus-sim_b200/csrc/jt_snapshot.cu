// Snapshot / checkpoint I/O in the reference's snapshot_v3 format
// (src/snapshot_v3.rs:12-47, 260-376), so that a run of this engine can be
// checkpointed, resumed, and read by the reference's own analysis tools.
//
// Layout (little-endian): a 408-byte header -- magic u64 "JANUSV3\n",
// version u32 = 3, header_size u32 = 408, n_total u64, then f64 a, t_gyr,
// l_box, h0, mu, omega_b, m_part_plus_base, m_part_minus_base,
// eps_plus_base, eps_minus_base, u32 n_split_max, u32 seed_ic, f64 z_init,
// u64 n_stars, f64 z_start_run, f64 sfr, f64 rho_max, u8 run_label[256] --
// followed by n_total 36-byte particles: f32 pos[3], f32 vel[3], f32 mass,
// f32 epsilon, u8 sign (1 = m+, 255 = m-), u8 split_level, u8 is_star,
// u8 flags.  Host code only (the device state is copied out by the caller
// entry point).
#include "jt_batch.h"

#include <cstdio>
#include <cstring>
#include <vector>

namespace {

constexpr uint64_t kMagic = 0x0A335653554E414AULL;   // "JANUSV3\n" read as little-endian u64
constexpr uint32_t kVersion = 3, kHeaderSize = 408, kParticleSize = 36;

struct Writer {
    std::vector<unsigned char> b;
    template <class T>
    void put(T v)
    {
        unsigned char tmp[sizeof(T)];
        std::memcpy(tmp, &v, sizeof(T));   // the hosts this library targets are little-endian
        b.insert(b.end(), tmp, tmp + sizeof(T));
    }
};

template <class T>
T get(const unsigned char*& p)
{
    T v;
    std::memcpy(&v, p, sizeof(T));
    p += sizeof(T);
    return v;
}

}  // namespace

extern "C" {

int jt_snapshot_write(const char* path, const jt_snapshot_meta* meta, double box_L, double mu,
                      const float* pos, const float* vel, const int8_t* signs, const float* mass,
                      const float* eps, size_t n)
{
    if (!path || !meta || (n && (!pos || !signs || !mass || !eps))) return JT_EINVAL;
    Writer w;
    float mp = 0.f, mm = 0.f, ep = 0.f, em = 0.f;
    for (size_t i = 0; i < n; i++) {
        if (signs[i] > 0 && mp == 0.f) { mp = mass[i]; ep = eps[i]; }
        if (signs[i] < 0 && mm == 0.f) { mm = mass[i]; em = eps[i]; }
    }
    w.put<uint64_t>(kMagic);
    w.put<uint32_t>(kVersion);
    w.put<uint32_t>(kHeaderSize);
    w.put<uint64_t>((uint64_t)n);
    w.put<double>(meta->a);
    w.put<double>(meta->t_gyr);
    w.put<double>(box_L);
    w.put<double>(meta->h0);
    w.put<double>(mu);
    w.put<double>(meta->omega_b);
    w.put<double>(mp);
    w.put<double>(mm);
    w.put<double>(ep);
    w.put<double>(em);
    w.put<uint32_t>(0);                 // n_split_max: no particle splitting here
    w.put<uint32_t>(meta->seed_ic);
    w.put<double>(meta->z_init);
    w.put<uint64_t>(0);                 // n_stars
    w.put<double>(meta->z_start_run);
    w.put<double>(0.0);                 // sfr
    w.put<double>(0.0);                 // rho_max
    unsigned char label[256] = {0};
    std::memcpy(label, meta->run_label, 255);
    w.b.insert(w.b.end(), label, label + 256);
    if (w.b.size() != kHeaderSize) return JT_EINVAL;
    FILE* f = std::fopen(path, "wb");
    if (!f) return JT_EINVAL;
    bool ok = std::fwrite(w.b.data(), 1, w.b.size(), f) == w.b.size();
    std::vector<unsigned char> rec;
    const size_t chunk = 1 << 16;
    rec.reserve(chunk * kParticleSize);
    for (size_t i0 = 0; i0 < n && ok; i0 += chunk) {
        const size_t i1 = std::min(n, i0 + chunk);
        rec.clear();
        Writer r;
        r.b.swap(rec);
        for (size_t i = i0; i < i1; i++) {
            for (int d = 0; d < 3; d++) r.put<float>(pos[3 * i + d]);
            for (int d = 0; d < 3; d++) r.put<float>(vel ? vel[3 * i + d] : 0.0f);
            r.put<float>(mass[i]);
            r.put<float>(eps[i]);
            r.put<uint8_t>(signs[i] > 0 ? 1 : 255);
            r.put<uint8_t>(0);
            r.put<uint8_t>(0);
            r.put<uint8_t>(0);
        }
        ok = std::fwrite(r.b.data(), 1, r.b.size(), f) == r.b.size();
        rec.swap(r.b);
    }
    ok = (std::fclose(f) == 0) && ok;
    return ok ? JT_OK : JT_EINVAL;
}

int jt_snapshot_read(const char* path, jt_snapshot_meta* meta, double* box_L, double* mu, float* pos,
                     float* vel, int8_t* signs, float* mass, float* eps, size_t cap, size_t* n)
{
    if (!path || !n) return JT_EINVAL;
    FILE* f = std::fopen(path, "rb");
    if (!f) return JT_EINVAL;
    unsigned char h[kHeaderSize];
    if (std::fread(h, 1, 16, f) != 16) {
        std::fclose(f);
        return JT_EINVAL;
    }
    const unsigned char* p = h;
    const uint64_t magic = get<uint64_t>(p);
    const uint32_t version = get<uint32_t>(p);
    const uint32_t hsize = get<uint32_t>(p);
    if (magic != kMagic || version != kVersion || hsize < kHeaderSize ||
        std::fread(h + 16, 1, kHeaderSize - 16, f) != kHeaderSize - 16) {
        std::fclose(f);
        return JT_EINVAL;
    }
    const uint64_t nt = get<uint64_t>(p);
    jt_snapshot_meta m;
    std::memset(&m, 0, sizeof(m));
    m.a = get<double>(p);
    m.t_gyr = get<double>(p);
    const double L = get<double>(p);
    m.h0 = get<double>(p);
    const double mu_ = get<double>(p);
    m.omega_b = get<double>(p);
    p += 4 * 8 + 4;                     // base masses and softenings, n_split_max
    m.seed_ic = get<uint32_t>(p);
    m.z_init = get<double>(p);
    p += 8;                             // n_stars
    m.z_start_run = get<double>(p);
    p += 16;                            // sfr, rho_max
    std::memcpy(m.run_label, p, 255);
    m.run_label[255] = 0;
    if (meta) *meta = m;
    if (box_L) *box_L = L;
    if (mu) *mu = mu_;
    *n = (size_t)nt;
    if (!pos) {                         // size query
        std::fclose(f);
        return JT_OK;
    }
    if (cap < nt || !signs) {
        std::fclose(f);
        return JT_EINVAL;
    }
    if (hsize > kHeaderSize) std::fseek(f, (long)hsize, SEEK_SET);
    std::vector<unsigned char> rec((size_t)kParticleSize << 16);
    const size_t chunk = 1 << 16;
    for (size_t i0 = 0; i0 < nt; i0 += chunk) {
        const size_t i1 = std::min((size_t)nt, i0 + chunk);
        const size_t bytes = (i1 - i0) * kParticleSize;
        if (std::fread(rec.data(), 1, bytes, f) != bytes) {
            std::fclose(f);
            return JT_EINVAL;
        }
        const unsigned char* q = rec.data();
        for (size_t i = i0; i < i1; i++) {
            for (int d = 0; d < 3; d++) pos[3 * i + d] = get<float>(q);
            for (int d = 0; d < 3; d++) {
                const float v = get<float>(q);
                if (vel) vel[3 * i + d] = v;
            }
            const float ms = get<float>(q), es = get<float>(q);
            if (mass) mass[i] = ms;
            if (eps) eps[i] = es;
            const uint8_t sg = get<uint8_t>(q);
            signs[i] = sg == 1 ? 1 : -1;
            q += 3;
        }
    }
    std::fclose(f);
    return JT_OK;
}

// Checkpoint a handle's state: positions and velocities in the caller's
// order (the signed array it was loaded with, or [m+ ; m-]), its signs, and
// per-particle mass and softening from the config.
int jt_checkpoint(jt_handle* h, const char* path, const jt_snapshot_meta* meta)
{
    if (!h || !path || !meta) return JT_EINVAL;
    size_t np = 0, nm = 0;
    int r = jt_counts(h, &np, &nm);
    if (r != JT_OK) return r;
    const size_t n = np + nm;
    if (n == 0) return JT_ESTATE;
    std::vector<float> pos(3 * n), vel(3 * n), mass(n), eps(n);
    std::vector<int8_t> sg(n);
    jt_config cfg;
    float mp = 0.f, mm = 0.f;
    if ((r = jth_info(h, &cfg, &mp, &mm, sg.data())) != JT_OK) return r;
    if ((r = jt_get_state_signed(h, pos.data(), vel.data(), JT_MEM_HOST)) != JT_OK) return r;
    for (size_t i = 0; i < n; i++) {
        mass[i] = sg[i] > 0 ? mp : mm;
        eps[i] = (float)cfg.softening;
    }
    return jt_snapshot_write(path, meta, cfg.box_L, cfg.mu, pos.data(), vel.data(), sg.data(), mass.data(),
                             eps.data(), n);
}

}  // extern "C"
