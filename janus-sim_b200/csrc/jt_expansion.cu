// FP64 Janus expansion history: the scale factor, cosmic time and Hubble rate
// of the positive sector that set the kick's drag factor (H in
// v += (a - H v dtau) dt) and the step schedule in time.
//
// The reference's JanusExpansion (src/janus_expansion.rs:62-266) is the
// exact parametric solution of the Janus positive sector, in units where
// H0 = 0.0715 / Gyr:
//   a+(mu) = alpha^2 cosh^2 mu,   t+(mu) = alpha^2 (mu + sinh^2(mu) / 2),
//   H+(mu) = sinh(2 mu) / (alpha^2 cosh^2 mu (1 + sinh(2 mu) / 2)),
// with mu0 = 1.5 and alpha^2 fixed by H+(mu0) = 1 (calibrate_alpha_mu0,
// :247-266), a normalised to 1 at mu0 and z = a0 / (alpha^2 cosh^2 mu) - 1.
// Every expression keeps the reference's operation order, so the states
// agree to the last bit where the host's libm does.
// Its drivers build a table of n states uniform in mu from z_init to z = 0
// (JanusExpansion::new, :62-123; the production run uses z_init = 4 and 5000
// rows, src/bin/janus_mu19_production.rs:46) and interpolate it linearly in
// time or redshift (at_time :126-154, at_redshift :157-180).  The same
// table, the same clamps and the same interpolation are kept here, so a
// driver calling jt_expansion_at_time gets the reference's numbers; the
// library prints nothing (the reference prints the table's summary and a
// warning when z_init is clamped; jt_expansion_info returns both).
//
// The cross-species factors of the eta parameter scans follow
// src/vsl_dynamic.rs:138-142 (a- = a+ (1 + z)^{-(eta - 1) / eta}) and
// src/janus_expansion.rs:449-462 (phi = (a- / a+)^3 and its inverse).
#include "jt_internal.cuh"

#include <algorithm>
#include <cmath>
#include <new>
#include <vector>

namespace {

constexpr double kH0GyrInv = 0.0715;   // H0 = 70 km/s/Mpc in 1/Gyr, as the reference
constexpr double kMu0 = 1.5;

jt_expansion_state state_at(double mu, double alpha, double a_0)
{
    const double c = std::cosh(mu), s = std::sinh(mu), s2 = std::sinh(2.0 * mu);
    const double a2 = alpha * alpha;
    const double a_raw = a2 * c * c;
    jt_expansion_state st;
    st.mu = mu;
    st.a_plus = a_raw / a_0;
    st.t_gyr = a2 * (mu + 0.5 * (s * s)) / kH0GyrInv;
    st.h_plus = s2 / (a2 * c * c * (1.0 + 0.5 * s2)) * kH0GyrInv;
    st.z = a_0 / a_raw - 1.0;
    return st;
}

void calibrate(double* alpha, double* mu_0)
{
    const double c = std::cosh(kMu0), s2 = std::sinh(2.0 * kMu0);
    *alpha = std::sqrt(s2 / (c * c * (1.0 + 0.5 * s2)));
    *mu_0 = kMu0;
}

jt_expansion_state lerp(const jt_expansion_state& s0, const jt_expansion_state& s1, double f)
{
    jt_expansion_state r;
    r.mu = s0.mu + f * (s1.mu - s0.mu);
    r.a_plus = s0.a_plus + f * (s1.a_plus - s0.a_plus);
    r.t_gyr = s0.t_gyr + f * (s1.t_gyr - s0.t_gyr);
    r.h_plus = s0.h_plus + f * (s1.h_plus - s0.h_plus);
    r.z = s0.z + f * (s1.z - s0.z);
    return r;
}

}  // namespace

struct jt_expansion {
    double alpha = 0, mu_0 = 0, a_0 = 0, z_max = 0, z_init = 0;
    std::vector<jt_expansion_state> table;
};

extern "C" int jt_expansion_calibrate(double* alpha, double* mu_0)
{
    if (!alpha || !mu_0) return JT_EINVAL;
    calibrate(alpha, mu_0);
    return JT_OK;
}

extern "C" int jt_expansion_state_at_mu(double mu, double alpha, double a_0, jt_expansion_state* out)
{
    if (!out || !std::isfinite(mu) || !(alpha > 0.0) || !(a_0 > 0.0)) return JT_EINVAL;
    *out = state_at(mu, alpha, a_0);
    return JT_OK;
}

extern "C" int jt_expansion_create(double z_init, int n_points, jt_expansion** out)
{
    if (!out) return JT_EINVAL;
    *out = nullptr;
    if (!(z_init >= 0.0) || !std::isfinite(z_init) || n_points < 2) return JT_EINVAL;
    jt_expansion* e = new (std::nothrow) jt_expansion;
    if (!e) return JT_ENOMEM;
    calibrate(&e->alpha, &e->mu_0);
    const double a2 = e->alpha * e->alpha;
    const double c0 = std::cosh(e->mu_0);
    e->a_0 = a2 * (c0 * c0);
    // the parametric solution bottoms out at mu = 0 (a = alpha^2)
    e->z_max = e->a_0 / a2 - 1.0;
    e->z_init = std::min(z_init, e->z_max * 0.99);
    const double a_init = e->a_0 / (1.0 + e->z_init);
    const double cosh_mu = std::max(std::sqrt(a_init / a2), 1.0);
    const double mu_init = std::acosh(cosh_mu);
    const double d_mu = (e->mu_0 - mu_init) / ((double)n_points - 1.0);
    try {
        e->table.resize((size_t)n_points);
    } catch (...) {
        delete e;
        return JT_ENOMEM;
    }
    for (int i = 0; i < n_points; i++) e->table[i] = state_at(mu_init + i * d_mu, e->alpha, e->a_0);
    *out = e;
    return JT_OK;
}

extern "C" void jt_expansion_destroy(jt_expansion* e) { delete e; }

extern "C" int jt_expansion_info(const jt_expansion* e, jt_expansion_info_t* out)
{
    if (!e || !out) return JT_EINVAL;
    out->alpha = e->alpha;
    out->mu_0 = e->mu_0;
    out->a_0 = e->a_0;
    out->z_max = e->z_max;
    out->z_init = e->z_init;
    out->t_start = e->table.front().t_gyr;
    out->t_end = e->table.back().t_gyr;
    out->n_points = (int64_t)e->table.size();
    return JT_OK;
}

extern "C" int jt_expansion_at_time(const jt_expansion* e, double t_gyr, jt_expansion_state* out)
{
    if (!e || !out || std::isnan(t_gyr)) return JT_EINVAL;
    const auto& T = e->table;
    const double t = std::min(std::max(t_gyr, T.front().t_gyr), T.back().t_gyr);
    // first row with t_gyr >= t (partition_point of t_gyr < t)
    const size_t idx = (size_t)(std::lower_bound(T.begin(), T.end(), t,
                                                 [](const jt_expansion_state& s, double v) {
                                                     return s.t_gyr < v;
                                                 }) - T.begin());
    if (idx == 0) { *out = T.front(); return JT_OK; }
    if (idx >= T.size()) { *out = T.back(); return JT_OK; }
    const auto& s0 = T[idx - 1];
    const auto& s1 = T[idx];
    *out = lerp(s0, s1, (t - s0.t_gyr) / (s1.t_gyr - s0.t_gyr));
    out->t_gyr = t;
    return JT_OK;
}

extern "C" int jt_expansion_at_redshift(const jt_expansion* e, double z, jt_expansion_state* out)
{
    if (!e || !out || std::isnan(z)) return JT_EINVAL;
    const auto& T = e->table;
    // first row with z <= the argument (z decreases along the table)
    const size_t idx = (size_t)(std::partition_point(T.begin(), T.end(),
                                                     [z](const jt_expansion_state& s) { return s.z > z; }) -
                                T.begin());
    if (idx == 0) { *out = T.front(); return JT_OK; }
    if (idx >= T.size()) { *out = T.back(); return JT_OK; }
    const auto& s0 = T[idx - 1];
    const auto& s1 = T[idx];
    *out = lerp(s0, s1, (s0.z - z) / (s0.z - s1.z));
    out->z = z;
    return JT_OK;
}

extern "C" int jt_expansion_phi_factors(double a_plus, double eta, double* a_minus, double* phi,
                                        double* phi_inv)
{
    if (!(a_plus > 0.0) || !(eta > 0.0) || !std::isfinite(a_plus) || !std::isfinite(eta)) return JT_EINVAL;
    const double z = 1.0 / a_plus - 1.0;
    const double am = a_plus * std::pow(1.0 + z, -(eta - 1.0) / eta);
    const double r = am / a_plus, ri = a_plus / am;
    if (a_minus) *a_minus = am;
    if (phi) *phi = r * r * r;
    if (phi_inv) *phi_inv = ri * ri * ri;
    return JT_OK;
}
