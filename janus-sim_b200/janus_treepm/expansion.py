"""Janus expansion history in FP64, through the library's jt_expansion_*.

The reference's JanusExpansion (janus-sim src/janus_expansion.rs:62-266):
the parametric positive-sector solution a+(mu) = alpha^2 cosh^2 mu,
t+(mu) = alpha^2 (mu + sinh^2(mu)/2) / H0, H+(mu) = H0 sinh(2 mu) /
(alpha^2 cosh^2 mu (1 + sinh(2 mu)/2)), H0 = 0.0715 / Gyr, mu0 = 1.5, tabulated
uniformly in mu from z_init to z = 0 and interpolated linearly in time or
redshift (at_time, at_redshift), as the reference's drivers use it
(src/bin/janus_mu19_production.rs:46, 119-137).
"""
import ctypes as C

from . import library, _check, jt_expansion_state, jt_expansion_info_t


class Expansion:
    """JanusExpansion::new(z_init, n_points)."""

    def __init__(self, z_init=4.0, n_points=5000):
        self._h = C.c_void_p()
        _check(library().jt_expansion_create(float(z_init), int(n_points), C.byref(self._h)),
               "jt_expansion_create")

    def close(self):
        if self._h:
            library().jt_expansion_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def info(self):
        o = jt_expansion_info_t()
        _check(library().jt_expansion_info(self._h, C.byref(o)), "jt_expansion_info")
        return {k: getattr(o, k) for k, _ in o._fields_}

    def at_time(self, t_gyr):
        o = jt_expansion_state()
        _check(library().jt_expansion_at_time(self._h, float(t_gyr), C.byref(o)), "jt_expansion_at_time")
        return o.to_dict()

    def at_redshift(self, z):
        o = jt_expansion_state()
        _check(library().jt_expansion_at_redshift(self._h, float(z), C.byref(o)), "jt_expansion_at_redshift")
        return o.to_dict()


def calibrate():
    """(alpha, mu_0) of calibrate_alpha_mu0."""
    a, m = C.c_double(), C.c_double()
    _check(library().jt_expansion_calibrate(C.byref(a), C.byref(m)), "jt_expansion_calibrate")
    return a.value, m.value


def state_at_mu(mu, alpha, a_0):
    """compute_state(mu, alpha, a_0) as a dict."""
    o = jt_expansion_state()
    _check(library().jt_expansion_state_at_mu(float(mu), float(alpha), float(a_0), C.byref(o)),
           "jt_expansion_state_at_mu")
    return o.to_dict()


def phi_factors(a_plus, eta):
    """(a_minus, phi, phi_inv) of the eta coupling."""
    am, p, pi = C.c_double(), C.c_double(), C.c_double()
    _check(library().jt_expansion_phi_factors(float(a_plus), float(eta), C.byref(am), C.byref(p),
                                              C.byref(pi)), "jt_expansion_phi_factors")
    return am.value, p.value, pi.value


def state_at_redshift(z, n_points=5000):
    """(a_plus, t_gyr, h_plus, z) at redshift z from a table that starts there
    (its first row: the exact state)."""
    e = Expansion(z, n_points)
    s = e.at_redshift(z)
    e.close()
    return s["a_plus"], s["t_gyr"], s["h_plus"], s["z"]
