"""The FP64 Janus expansion (jt_expansion_*) against the reference's formulas.

The expected values are computed here from src/janus_expansion.rs restated
in plain Python (math: the same libm as the library), operation for
operation: calibrate_alpha_mu0 (:247-266), compute_state (:196-230),
JanusExpansion::new (:62-123), at_time (:126-154), at_redshift (:157-180);
and the eta coupling (src/vsl_dynamic.rs:138-142, janus_expansion.rs:449-462).
Also the reference's own known answers: H(z = 0) = 70 km/s/Mpc to 1
(test_calibration), a decreasing with z and <= 1 (test_redshift_evolution),
phi = 1 at z = 0 (test_phi_convergence_at_z0).  No GPU needed.
"""
import bisect
import math

import numpy as np

from janus_treepm import expansion as E

H0 = 0.0715
KM_S_MPC_TO_GYR_INV = 1.0227e-3


def _calibrate():
    mu0 = 1.5
    c = math.cosh(mu0)
    s2 = math.sinh(2.0 * mu0)
    return math.sqrt(s2 / (c * c * (1.0 + 0.5 * s2))), mu0


def _state(mu, alpha, a0):
    c, s, s2 = math.cosh(mu), math.sinh(mu), math.sinh(2.0 * mu)
    a_raw = alpha * alpha * c * c
    return {"mu": mu, "a_plus": a_raw / a0, "t_gyr": alpha * alpha * (mu + 0.5 * (s * s)) / H0,
            "h_plus": s2 / (alpha * alpha * c * c * (1.0 + 0.5 * s2)) * H0, "z": a0 / a_raw - 1.0}


def _table(z_init, n):
    alpha, mu0 = _calibrate()
    a0 = alpha * alpha * (math.cosh(mu0) ** 2)
    z_max = a0 / (alpha * alpha) - 1.0
    zc = min(z_init, z_max * 0.99)
    a_init = a0 / (1.0 + zc)
    mu_init = math.acosh(max(math.sqrt(a_init / (alpha * alpha)), 1.0))
    d = (mu0 - mu_init) / (n - 1.0)
    return [_state(mu_init + i * d, alpha, a0) for i in range(n)], alpha, mu0, a0, z_max, zc


def _lerp(s0, s1, f):
    return {k: s0[k] + f * (s1[k] - s0[k]) for k in s0}


def _at_time(tab, t):
    t = min(max(t, tab[0]["t_gyr"]), tab[-1]["t_gyr"])
    i = bisect.bisect_left([s["t_gyr"] for s in tab], t)
    if i == 0:
        return tab[0]
    if i >= len(tab):
        return tab[-1]
    s0, s1 = tab[i - 1], tab[i]
    r = _lerp(s0, s1, (t - s0["t_gyr"]) / (s1["t_gyr"] - s0["t_gyr"]))
    r["t_gyr"] = t
    return r


def _at_redshift(tab, z):
    i = 0
    while i < len(tab) and tab[i]["z"] > z:
        i += 1
    if i == 0:
        return tab[0]
    if i >= len(tab):
        return tab[-1]
    s0, s1 = tab[i - 1], tab[i]
    r = _lerp(s0, s1, (s0["z"] - z) / (s0["z"] - s1["z"]))
    r["z"] = z
    return r


def _close(a, b, tol=1e-14):
    for k in b:
        assert abs(a[k] - b[k]) <= tol * max(1.0, abs(b[k])), (k, a[k], b[k])


def test_calibration_and_state():
    alpha, mu0 = E.calibrate()
    ra, rm = _calibrate()
    assert alpha == ra and mu0 == rm
    a0 = alpha * alpha * math.cosh(mu0) ** 2
    for mu in (0.0, 0.3, 0.79, 1.2, 1.5):
        _close(E.state_at_mu(mu, alpha, a0), _state(mu, alpha, a0))


def test_table_and_interpolation_match_the_reference():
    for z_init, n in ((4.0, 5000), (10.0, 2000), (5.0, 1000)):
        tab, alpha, mu0, a0, z_max, zc = _table(z_init, n)
        e = E.Expansion(z_init, n)
        info = e.info()
        assert info["n_points"] == n
        for k, v in (("alpha", alpha), ("mu_0", mu0), ("a_0", a0), ("z_max", z_max), ("z_init", zc),
                     ("t_start", tab[0]["t_gyr"]), ("t_end", tab[-1]["t_gyr"])):
            assert abs(info[k] - v) <= 1e-14 * abs(v), (k, info[k], v)
        rng = np.random.default_rng(3)
        ts = list(rng.uniform(tab[0]["t_gyr"] - 1.0, tab[-1]["t_gyr"] + 1.0, 200)) + \
            [tab[0]["t_gyr"], tab[-1]["t_gyr"], tab[7]["t_gyr"]]
        for t in ts:
            _close(e.at_time(t), _at_time(tab, t))
        for z in list(rng.uniform(-0.5, zc + 1.0, 200)) + [0.0, zc, tab[9]["z"]]:
            _close(e.at_redshift(z), _at_redshift(tab, z))
        e.close()


def test_reference_known_answers():
    # test_calibration: H(z = 0) = 70 km/s/Mpc to 1
    e = E.Expansion(5.0, 1000)
    h0 = e.at_redshift(0.0)["h_plus"] / KM_S_MPC_TO_GYR_INV
    assert abs(h0 - 70.0) < 1.0, h0
    e.close()
    # test_redshift_evolution: a decreases with z and stays <= 1
    e = E.Expansion(10.0, 2000)
    a = [e.at_redshift(z)["a_plus"] for z in (0.0, 1.0, 2.0, 5.0, 10.0)]
    assert all(x > 0.0 for x in a) and a[0] <= 1.0 + 1e-12
    assert all(a[i] > a[i + 1] for i in range(len(a) - 1)) or a[-1] == a[-2]
    e.close()
    # z_init beyond the parametric limit is clamped to 0.99 z_max
    e = E.Expansion(50.0, 100)
    info = e.info()
    assert abs(info["z_init"] - 0.99 * info["z_max"]) <= 1e-12 * info["z_max"]
    e.close()


def test_eta_coupling():
    for a_plus, eta in ((1.0, 1.045), (0.2, 1.045), (0.5, 1.1), (0.33, 1.0)):
        z = 1.0 / a_plus - 1.0
        am = a_plus * (1.0 + z) ** (-(eta - 1.0) / eta)
        got = E.phi_factors(a_plus, eta)
        assert abs(got[0] - am) <= 1e-15 * am
        assert abs(got[1] - (am / a_plus) ** 3) <= 1e-14
        assert abs(got[2] - (a_plus / am) ** 3) <= 1e-14
    # test_phi_convergence_at_z0: phi = 1 at z = 0
    assert abs(E.phi_factors(1.0, 1.045)[1] - 1.0) < 1e-12
