"""FP64 energy diagnostics on the device (jt_energy_sampled,
jt_virialize_sampled) against the oracle's restatement of the reference's
host-side kinetic_energy / potential_energy_binding_sampled /
virialize_sampled (src/nbody_gpu_twopass.rs:5070-5225); energy_drift_pct on
the host.  Tolerance 1e-10 relative (FP64 sums in a different order)."""
import os
import sys

import numpy as np
import pytest

import janus_treepm as J

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402


def test_energy_drift_pct():
    assert J.energy_drift_pct(-99.0, -100.0) == pytest.approx(1.0)
    assert J.energy_drift_pct(110.0, 100.0) == pytest.approx(10.0)
    assert J.energy_drift_pct(5.0, 1e-31) == 0.0


def test_oracle_pe_small_case():
    pp = np.array([[0, 0, 0], [3, 4, 0], [0, 0, 1]], np.float64)
    pe, _ = O.pe_binding_sampled(pp, np.zeros((0, 3)), 10, 0.0)
    assert pe == pytest.approx(-(1 / 5 + 1 + 1 / np.sqrt(9 + 16 + 1)))


def _state(n_p, n_m, L, seed):
    rng = np.random.default_rng(seed)
    pp = ((rng.random((n_p, 3)) - 0.5) * L).astype(np.float32)
    pm = ((rng.random((n_m, 3)) - 0.5) * L).astype(np.float32)
    vp = rng.normal(0, 0.3, (n_p, 3)).astype(np.float32)
    vm = rng.normal(0, 0.3, (n_m, 3)).astype(np.float32)
    return pp, vp, pm, vm


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 1])
@pytest.mark.parametrize("n_sample", [700, 5000])
def test_energy_matches_oracle(mode, n_sample):
    L, eps = 40.0, 0.07
    pp, vp, pm, vm = _state(3001, 2200, L, 3)
    s = J.Solver(J.Config(box_L=L, pm_grid=32, softening=eps, mu=4.0, mode=mode))
    s.set_state(pp, vp, pm, vm)
    e = s.energy(n_sample)
    ke = O.kinetic_energy_unit(vp, vm)
    pe_p, pe_m = O.pe_binding_sampled(pp, pm, n_sample, eps)
    assert e["kinetic"] == pytest.approx(ke, rel=1e-10)
    assert e["pe_plus"] == pytest.approx(pe_p, rel=1e-10)
    assert e["pe_minus"] == pytest.approx(pe_m, rel=1e-10)
    assert e["n_sampled"] == (min(3001, n_sample), min(2200, n_sample))
    s.close()


@pytest.mark.gpu
def test_virialize_scales_to_the_virial_ratio():
    L, eps = 20.0, 0.05
    pp, vp, pm, vm = _state(1500, 1500, L, 8)
    s = J.Solver(J.Config(box_L=L, pm_grid=16, softening=eps, mu=1.0))
    s.set_state(pp, vp, pm, vm)
    alpha = s.virialize(1000)
    pe_p, pe_m = O.pe_binding_sampled(pp, pm, 1000, eps)
    ke = O.kinetic_energy_unit(vp, vm)
    assert alpha == pytest.approx(np.sqrt(abs(pe_p + pe_m) / 2.0 / ke), rel=1e-10)
    gp, gvp, gm, gvm = s.get_state()
    assert np.array_equal(gvp, (vp * np.float32(alpha)).astype(np.float32))
    assert np.array_equal(gp, pp)
    e = s.energy(1000)
    assert 2.0 * e["kinetic"] == pytest.approx(abs(e["pe_binding"]), rel=1e-6)
    s.close()
