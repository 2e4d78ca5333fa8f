"""The fused z transforms + k-space kernel of 512^3 and 256^3 grids (jt_zfft.cu) against
the 3D path it replaces (cuFFT 3D R2C, k_b_kspace, cuFFT 3D C2R; selected
with JT_ZFFT=0 when a handle is made).

Both paths compute the same long-range forces up to float rounding of two
FFT factorisations; the test asks for agreement to 1e-5 of the rms PM force
(float FFTs of 512^3 grids agree to a few 1e-7), with interlaced and single
grids, k_min, and the screened split (two sources, the unsigned one through
the second launch)."""
import os

import numpy as np
import pytest

import janus_treepm as J
from janus_treepm import ics

pytestmark = pytest.mark.gpu


def _pm(cfg, pp, pm, fused, screening=None):
    # the choice is read when the handle's first pass makes its grid bucket
    old = os.environ.get("JT_ZFFT")
    os.environ["JT_ZFFT"] = "1" if fused else "0"
    try:
        s = J.Solver(cfg)
        s.set_state(pp, None, pm, None)
        if screening is not None:
            s.set_screening(*screening)
        ap, am = s.accel_part(J.JT_PART_PM)
        s.close()
    finally:
        if old is None:
            del os.environ["JT_ZFFT"]
        else:
            os.environ["JT_ZFFT"] = old
    return np.concatenate([ap, am]).astype(np.float64)


def _check(a, b, tol=1e-5):
    rms = np.sqrt(np.mean(np.sum(b * b, axis=1)))
    err = np.abs(a - b).max() / rms
    assert np.all(np.isfinite(a)) and err <= tol, err


@pytest.mark.parametrize("M,interlace,k_min", [(512, 0, 0), (512, 2, 0), (512, 0, 3), (256, 0, 0), (256, 2, 3)])
def test_fused_z_transforms_match_the_3d_path(M, interlace, k_min):
    L, n = 200.0 * M / 512, 48
    pp, _, pm, _ = ics.zeldovich_lattice(n, L, seed=7)
    cfg = J.Config(box_L=L, pm_grid=M, theta=0.5, softening=0.02, r_s=1.25 * L / M, r_cut=4.5 * 1.25 * L / M,
                   mu=19.0, G_mass_plus=1e-3, mode=J.JT_ACCURATE, pm_interlace=interlace, k_min=k_min)
    _check(_pm(cfg, pp, pm, True), _pm(cfg, pp, pm, False))


@pytest.mark.parametrize("M", [512, 256])
def test_fused_z_transforms_screened(M):
    L, n = 150.0 * M / 512, 40
    pp, pm = ics.uniform_box(n ** 3, L, seed=3)
    cfg = J.Config(box_L=L, pm_grid=M, theta=0.5, softening=0.02, r_s=1.25 * L / M, r_cut=4.5 * 1.25 * L / M,
                   mu=19.0, G_mass_plus=1e-3, mode=J.JT_ACCURATE)
    _check(_pm(cfg, pp, pm, True, (5.0, 0.5)), _pm(cfg, pp, pm, False, (5.0, 0.5)))
