"""Device diagnostics (jt_diagnostics / jt_batch_diagnostics) against numpy
restatements of the reference's host-side metrics (oracle/oracle.py:
segregation, segregation_metrics) and of the kinetic energy and momentum.
FP64 accumulation in a different order: relative tolerance 1e-9 (the NGP
cell counts are integers and must match exactly, so the grid metrics agree
to rounding)."""
import os
import sys

import numpy as np
import pytest

import janus_treepm as J

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
pytestmark = pytest.mark.gpu
TOL = 1e-9


def _check(d, pp, vp, pm, vm, L, n_cells, mass):
    import oracle as O
    pos = np.concatenate([pp, pm])
    sg = np.concatenate([np.ones(len(pp), np.int8), -np.ones(len(pm), np.int8)])
    assert abs(d["segregation"] - O.segregation(pos, sg, L)) <= TOL * max(1e-12, abs(d["segregation"])) + 1e-15
    dop, corr, exc = O.segregation_metrics(pos, sg, L, n_cells)
    assert d["diff_over_poisson"] == pytest.approx(dop, rel=TOL, abs=1e-12)
    assert d["corr"] == pytest.approx(corr, rel=TOL, abs=1e-12)
    assert d["exc_var_minus"] == pytest.approx(exc, rel=TOL, abs=1e-12)
    for s, (p, v) in enumerate(((pp, vp), (pm, vm))):
        v64 = v.astype(np.float64)
        ke = 0.5 * float(mass[s]) * float(np.sum(v64 * v64))
        mom = float(mass[s]) * v64.sum(axis=0)
        assert d["kinetic"][s] == pytest.approx(ke, rel=TOL)
        assert np.allclose(d["momentum"][s], mom, rtol=TOL, atol=1e-9 * np.abs(mom).max())
        assert np.allclose(d["com"][s], p.astype(np.float64).mean(axis=0), rtol=TOL, atol=1e-12)


def test_diagnostics_match_reference_metrics_before_and_after_steps():
    rng = np.random.default_rng(9)
    L, n_p, n_m = 80.0, 30000, 17000
    pp = rng.uniform(-L / 2, L / 2, (n_p, 3)).astype(np.float32)
    pm = np.concatenate([rng.uniform(-L / 2, 0, (n_m // 2, 3)),
                         rng.uniform(0, L / 2, (n_m - n_m // 2, 3))]).astype(np.float32)
    vp = rng.normal(0, 1, (n_p, 3)).astype(np.float32)
    vm = rng.normal(0, 1, (n_m, 3)).astype(np.float32)
    cfg = J.Config(box_L=L, pm_grid=64, mu=5.0, G_mass_plus=2.0, softening=0.05)
    s = J.Solver(cfg)
    s.set_state(pp, vp, pm, vm)
    mass = (2.0, np.float32(5.0 * 2.0 * n_p / n_m))
    _check(s.diagnostics(16), pp, vp, pm, vm, L, 16, mass)
    s.step(0.01, 0.0, 1.0, 2)
    a, b, c, d = s.get_state()
    _check(s.diagnostics(24), a, b, c, d, L, 24, mass)
    s.close()
    B = J.Batch()
    bid = B.add(cfg, pp, vp, pm, vm)
    _check(B.diagnostics(bid, 16), pp, vp, pm, vm, L, 16, mass)
    B.close()
