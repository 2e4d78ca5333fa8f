"""Janus expansion history in FP64 (the kick's Hubble drag factor).

Restates src/janus_expansion.rs (janus-sim): the parametric positive-sector
solution a+(mu) = alpha^2 cosh^2 mu, t+(mu) = alpha^2 (mu + sinh^2(mu)/2),
H+(mu) = sinh(2 mu) / (alpha^2 cosh^2 mu (1 + sinh(2 mu)/2)) in units of
H0 = 0.0715 / Gyr (compute_state :196-230), with alpha calibrated so that
H(mu0 = 1.5) = H0 (calibrate_alpha_mu0 :247-266) and z = a0 / a+ - 1.
"""
import math

H0_GYR_INV = 0.0715
MU0 = 1.5


def calibrate():
    s2 = math.sinh(2 * MU0)
    c = math.cosh(MU0)
    alpha_sq = s2 / (c * c * (1.0 + 0.5 * s2))
    a0 = alpha_sq * c * c
    return alpha_sq, a0


def state_at_mu(mu):
    """(a_plus (a0 = 1), t_gyr, h_plus [1/Gyr], z) at parameter mu."""
    alpha_sq, a0 = calibrate()
    c, s = math.cosh(mu), math.sinh(mu)
    s2 = math.sinh(2 * mu)
    a_raw = alpha_sq * c * c
    t = alpha_sq * (mu + 0.5 * s * s) / H0_GYR_INV
    h = s2 / (alpha_sq * c * c * (1.0 + 0.5 * s2)) * H0_GYR_INV
    return a_raw / a0, t, h, a0 / a_raw - 1.0


def state_at_redshift(z):
    """Exact inversion z -> mu (the reference interpolates a 5000-row table)."""
    alpha_sq, a0 = calibrate()
    a = a0 / (1.0 + z)
    cosh_mu = max(math.sqrt(a / alpha_sq), 1.0)
    return state_at_mu(math.acosh(cosh_mu))
