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


def test_checkpoint_and_resume(tmp_path):
    """Checkpoint after two steps, resume from the snapshot in a new handle,
    take two more steps; compare with the run that never stopped (resuming
    recomputes the forces at the same positions: velocities within 1e-5 of
    rms, positions within 1e-6 L)."""
    rng = np.random.default_rng(4)
    L, n = 60.0, 20000
    pos = rng.uniform(-L / 2, L / 2, (n, 3)).astype(np.float32)
    vel = rng.normal(0, 0.5, (n, 3)).astype(np.float32)
    sg = np.where(rng.random(n) < 0.5, 1, -1).astype(np.int8)
    cfg = J.Config(box_L=L, pm_grid=32, softening=0.05, mu=3.0)
    a = J.Solver(cfg)
    a.set_state_signed(pos, vel, sg)
    a.step(0.01, 0.05, 1.0, 2)
    path = tmp_path / "ck.bin"
    a.checkpoint(path, J.snapshot_meta(run_label="resume test"))
    a.step(0.01, 0.05, 1.0, 2)
    ref_p, ref_v = a.get_state()
    a.close()
    meta, L2, mu2, p, v, s, m, e = J.snapshot_read(path)
    assert L2 == L and mu2 == 3.0 and np.array_equal(s, sg) and meta.run_label == b"resume test"
    b = J.Solver(cfg)
    b.set_state_signed(p, v, s)
    b.step(0.01, 0.05, 1.0, 2)
    got_p, got_v = b.get_state()
    b.close()
    d = np.abs(got_p.astype(np.float64) - ref_p)
    d = np.minimum(d, L - d)
    assert d.max() <= 1e-6 * L
    rms = np.sqrt(np.mean(np.sum(ref_v.astype(np.float64) ** 2, axis=1)))
    assert np.abs(got_v.astype(np.float64) - ref_v).max() <= 1e-5 * rms
