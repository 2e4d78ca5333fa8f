"""GPU parity through the C ABI (janus-sim_b200/libjanus_treepm.so).

Bars:
  * Morton codes, sort permutation and LBVH topology: bit-exact against the
    oracle restatement of the reference build (pinned to the reference's own
    kernels in tests/test_oracle.py);
  * compatibility-mode accelerations against the oracle restatement of the
    reference's GPU forces: p99 relative error <= 1e-5 (the engine evaluates
    the same float expressions; the PM runs in FP32 where the reference runs
    FP64, and CUDA's erfcf differs from the host's by an ulp);
  * accurate-mode accelerations (PCS + interlacing, the default) against the
    FP64 exact split-model sum (same r_s, softening and r_cut, no grid, no
    tree): median <= 2e-4 and p99 <= 3e-3 at theta = 0.5 (the remaining error
    is the PM grid's; measured p50 8e-5, p99 1.3e-3 at 2x32^3 particles);
  * the m- response is the exact sign flip of the m+ response (bitwise).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mods():
    import janus_treepm as J
    import oracle as O
    return J, O


def _rel(a, b):
    return np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-30)


def _uniform(n, L, seed):
    rng = np.random.default_rng(seed)
    return ((rng.random((n, 3)) - 0.5) * L).astype(np.float32)


@pytest.mark.parametrize("n_p,n_m,collide", [(5000, 3001, False), (4096, 4096, True),
                                             (1, 2, False), (33, 0, False)])
def test_tree_topology_bitexact(n_p, n_m, collide):
    J, O = _mods()
    L = 64.0
    pp = _uniform(n_p, L, 1)
    pm = _uniform(n_m, L, 2)
    if collide:
        # many particles per 10-bit Morton cell: exercises the index tie-break
        cell = L / 1024
        pp = ((np.floor(pp / (128 * cell)) + 0.3) * 128 * cell).astype(np.float32)
        pm = ((np.floor(pm / (128 * cell)) + 0.6) * 128 * cell).astype(np.float32)
    s = J.Solver(J.Config(box_L=L, pm_grid=32, mode=J.JT_ACCURATE))
    s.set_state(pp, None, pm if n_m else None, None)
    for sp, pos in ((0, pp), (1, pm)):
        n = len(pos)
        if n == 0:
            continue
        got = s.debug_tree(sp)
        ref = O.build_tree(pos, np.float32(L / 2), 1.0)
        assert np.array_equal(got["morton"], ref["m30"])
        assert np.array_equal(got["perm"], ref["perm"])
        if n > 1:
            assert np.array_equal(got["left"][:n - 1], ref["left"][:n - 1])
            assert np.array_equal(got["right"][:n - 1], ref["right"][:n - 1])
        assert np.array_equal(got["parent"][:2 * n - 1], ref["parent"][:2 * n - 1])
    s.close()


@pytest.mark.parametrize("n,M,L,interleave", [(2048, 32, 64.0, False), (3000, 32, 50.0, True)])
def test_rcompat_matches_reference_forces(n, M, L, interleave):
    J, O = _mods()
    rng = np.random.default_rng(7)
    pos = _uniform(n, L, 3)
    if interleave:
        sg = np.where(rng.random(n) < 0.4, 1, -1).astype(np.int8)
    else:
        sg = np.concatenate([np.ones(n // 2, np.int8), -np.ones(n - n // 2, np.int8)])
    theta, eps, r_cut, mf = 0.5, 0.052913, 5.625, 0.01
    s = J.Solver(J.Config(box_L=L, pm_grid=M, theta=theta, softening=eps, r_s=r_cut / 3,
                          r_cut=r_cut, mu=(sg < 0).sum() / (sg > 0).sum(), G_mass_plus=mf,
                          mode=J.JT_RCOMPAT))
    s.set_state_signed(pos, None, sg)
    got = s.accel()
    ref = O.ref_total_forces(pos, sg, M, L, theta, eps, r_cut, mf)
    rel = _rel(got, ref)
    assert np.percentile(rel, 99) <= 1e-5, np.percentile(rel, [50, 99, 100])
    assert rel.max() <= 1e-3
    s.close()


@pytest.mark.parametrize("n,lam,z,theta,eps", [(2048, 1.93, 0.8, 0.5497, 0.0508),
                                               (3000, 0.35, 0.0, 0.7, 0.1),
                                               (1500, 7000.0, 9.0, 0.45, 0.02)])
def test_rcompat_screened_matches_reference_forces(n, lam, z, theta, eps):
    """Yukawa-screened walk (lambda_0 > 0.01) + PM against the oracle of the
    reference's screened branch; same bars as the unscreened case (CUDA's
    expf differs from the host's by an ulp or two)."""
    J, O = _mods()
    L, M, r_cut, mf = 40.0, 32, 5.0, 0.01
    rng = np.random.default_rng(17)
    pos = _uniform(n, L, 5)
    sg = np.where(rng.random(n) < 0.45, 1, -1).astype(np.int8)
    s = J.Solver(J.Config(box_L=L, pm_grid=M, theta=theta, softening=eps, r_s=r_cut / 3,
                          r_cut=r_cut, mu=(sg < 0).sum() / (sg > 0).sum(), G_mass_plus=mf,
                          mode=J.JT_RCOMPAT))
    s.set_state_signed(pos, None, sg)
    s.set_screening(lam, z)
    got = s.accel()
    ref = O.ref_total_forces_screened(pos, sg, M, L, theta, eps, r_cut, mf, lam, z)
    rel = _rel(got, ref)
    assert np.percentile(rel, 99) <= 1e-5, np.percentile(rel, [50, 99, 100])
    assert rel.max() <= 1e-3
    # off again: the erfc-split walk, as before
    s.set_screening(0.0, z)
    rel0 = _rel(s.accel(), O.ref_total_forces(pos, sg, M, L, theta, eps, r_cut, mf))
    assert np.percentile(rel0, 99) <= 1e-5
    s.close()


@pytest.mark.parametrize("lam,z,mu,cells", [(2.0, 0.0, 19.0, "1"), (0.6, 1.5, 1.0, "1"),
                                            (2.0, 0.0, 19.0, "0")])
def test_accurate_screened_matches_exact_split_model(lam, z, mu, cells):
    """Accurate mode with Yukawa screening of opposite-species pairs (kappa =
    1 / (lambda_0 sqrt(1 + z))) against the FP64 screened split sum (Ewald
    summation of both kernels) at the same r_cut, on 400 sampled targets;
    the near field through the cell walk and, with JT_WALK_CELLS=0, through
    the tree walk (no multipoles across species).  Same bars as the
    unscreened test."""
    import os
    J, O = _mods()
    n, M, L = 4096, 32, 32.0
    pp = _uniform(n, L, 11)
    pm = _uniform(n, L, 12)
    r_s = 1.25 * L / M
    r_cut = 4.5 * r_s
    eps = (L / (2 * n) ** (1 / 3)) / 30
    os.environ["JT_WALK_CELLS"] = cells
    try:
        s = J.Solver(J.Config(box_L=L, pm_grid=M, theta=0.5, softening=eps, r_s=r_s, r_cut=r_cut,
                              mu=mu, G_mass_plus=1.0, mode=J.JT_ACCURATE))
        s.set_screening(lam, z)   # before the state: kept when the box is made
        s.set_state(pp, None, pm, None)
        ap, am = s.accel()
        s.set_screening(0.0, 0.0)
        bp, bm = s.accel()
        s.close()
    finally:
        os.environ.pop("JT_WALK_CELLS", None)
    pos = np.concatenate([pp, pm]).astype(np.float64)
    mass = np.concatenate([np.full(n, 1.0), np.full(n, mu)])
    sg = np.concatenate([np.ones(n, np.int8), -np.ones(n, np.int8)])
    idx = np.random.default_rng(5).choice(2 * n, 400, replace=False)
    kappa = 1.0 / (lam * np.sqrt(1.0 + z))
    ex = O.ewald_forces_screened(pos, mass, sg, L, r_s, eps, kappa, r_trunc=r_cut, idx=idx)
    got = np.concatenate([ap, am])[idx]
    rel = _rel(got, ex)
    p50, p99 = np.percentile(rel, [50, 99])
    assert p99 <= 3e-3 and p50 <= 2e-4, (p50, p99)
    # screening changes the forces well beyond that error (the repulsion of
    # the other species is cut off beyond lambda)
    ex0 = O.ewald_forces_screened(pos, mass, sg, L, r_s, eps, 0.0, r_trunc=r_cut, idx=idx)
    assert np.median(_rel(ex0, ex)) > 0.05
    rel0 = _rel(np.concatenate([bp, bm])[idx], ex0)
    assert np.percentile(rel0, 99) <= 3e-3


def test_accurate_screening_limits():
    """A screening length far beyond the box is the unscreened model (to
    FP32 rounding of the extra terms), and lambda_0 <= 0.01 turns it off."""
    J, O = _mods()
    n, L = 3000, 40.0
    pp = _uniform(n, L, 31)
    pm = _uniform(n, L, 32)
    s = J.Solver(J.Config(box_L=L, pm_grid=32, mu=2.0, G_mass_plus=1.0, mode=J.JT_ACCURATE))
    s.set_state(pp, None, pm, None)
    a0 = np.concatenate(s.accel())
    s.set_screening(1.0e7, 0.0)
    a1 = np.concatenate(s.accel())
    rms = float(np.sqrt(np.mean(np.sum(a0.astype(np.float64) ** 2, axis=1))))
    d = np.linalg.norm(a1.astype(np.float64) - a0, axis=1) / rms
    assert np.percentile(d, 99) <= 2e-5 and d.max() <= 2e-4, (np.percentile(d, 99), d.max())
    s.set_screening(0.005, 0.0)
    a2 = np.concatenate(s.accel())
    d2 = np.linalg.norm(a2.astype(np.float64) - a0, axis=1) / rms
    assert np.percentile(d2, 99) <= 2e-5
    with pytest.raises(J.JanusError):
        s.set_screening(-1.0, 0.0)
    with pytest.raises(J.JanusError):
        s.set_screening(2.0, -1.0)
    s.close()


@pytest.mark.parametrize("n,M,L,mu", [(4096, 32, 32.0, 19.0), (8192, 64, 64.0, 1.0)])
def test_accurate_matches_exact_split_model(n, M, L, mu):
    J, O = _mods()
    pp = _uniform(n, L, 11)
    pm = _uniform(n, L, 12)
    r_s = 1.25 * L / M
    r_cut = 4.5 * r_s
    eps = (L / (2 * n) ** (1 / 3)) / 30
    s = J.Solver(J.Config(box_L=L, pm_grid=M, theta=0.5, softening=eps, r_s=r_s, r_cut=r_cut,
                          mu=mu, G_mass_plus=1.0, mode=J.JT_ACCURATE))
    s.set_state(pp, None, pm, None)
    ap, am = s.accel()
    pos = np.concatenate([pp, pm]).astype(np.float64)
    mass = np.concatenate([np.full(n, 1.0), np.full(n, mu)])
    sg = np.concatenate([np.ones(n, np.int8), -np.ones(n, np.int8)])
    ex = O.ewald_forces(pos, mass, sg, L, r_s, eps, r_trunc=r_cut)
    rel = _rel(np.concatenate([ap, am]), ex)
    p50, p99 = np.percentile(rel, [50, 99])
    assert p99 <= 3e-3 and p50 <= 2e-4, (p50, p99)
    s.close()


def test_cell_walk_wide_cut_without_softening():
    """A cut past 16 r_s, where the pair table ends (the split factor is below
    1e-27 there), and zero softening: the cell walk bounds its cut and its
    table index instead of clamping each pair's, and still matches the exact
    split model (5 cells per axis of 33 particles: every target takes the cell
    walk)."""
    J, O = _mods()
    n, M, L, mu = 2048, 128, 64.0, 19.0
    pp = _uniform(n, L, 21)
    pm = _uniform(n, L, 22)
    r_s = 1.25 * L / M
    r_cut = 20.0 * r_s
    s = J.Solver(J.Config(box_L=L, pm_grid=M, theta=0.5, softening=0.0, r_s=r_s, r_cut=r_cut,
                          mu=mu, G_mass_plus=1.0, mode=J.JT_ACCURATE))
    s.set_counters(True)
    s.set_state(pp, None, pm, None)
    ap, am = s.accel()
    t = s.timings()
    s.close()
    assert t["cellwalk_ms"] > 0.0 and t["node_interactions"] == 0, t
    pos = np.concatenate([pp, pm]).astype(np.float64)
    mass = np.concatenate([np.full(n, 1.0), np.full(n, mu)])
    sg = np.concatenate([np.ones(n, np.int8), -np.ones(n, np.int8)])
    ex = O.ewald_forces(pos, mass, sg, L, r_s, 0.0, r_trunc=r_cut)
    rel = _rel(np.concatenate([ap, am]), ex)
    p50, p99 = np.percentile(rel, [50, 99])
    assert p99 <= 3e-3 and p50 <= 2e-4, (p50, p99)


def test_minus_response_is_exact_sign_flip():
    J, O = _mods()
    n, L = 3000, 40.0
    pp = _uniform(n, L, 5)
    s = J.Solver(J.Config(box_L=L, pm_grid=32, mu=1.0, mode=J.JT_ACCURATE))
    s.set_state(pp, None, pp.copy(), None)
    ap, am = s.accel()
    assert np.array_equal(am, -ap)
    s.close()


def test_kdk_steps_repeat_within_rounding():
    """Three KDK steps twice from the same state agree to FP32 rounding (the
    deposit sums with float atomics, whose order varies run to run)."""
    J, O = _mods()
    n, L, mu = 4096, 32.0, 3.0
    pp = _uniform(n, L, 21)
    pm = _uniform(n, L, 22)
    s = J.Solver(J.Config(box_L=L, pm_grid=32, mu=mu, G_mass_plus=1e-3, mode=J.JT_ACCURATE))
    s.set_state(pp, None, pm, None)
    s.step(0.01, 0.0, 1.0, 3)
    a1 = s.get_state()
    s.set_state(pp, None, pm, None)
    s.step(0.01, 0.0, 1.0, 3)
    a2 = s.get_state()
    for x, y in zip(a1, a2):
        assert np.isfinite(x).all()
        assert np.abs(x - y).max() <= 1e-5 * max(np.abs(y).max(), 1e-12)
    s.close()


def test_kdk_matches_host_integration_of_device_forces():
    """One KDK step equals kick/drift applied on the host to jt_accel's
    accelerations (v += a dt/2; x += v dt; wrap; v += a' dt/2)."""
    J, O = _mods()
    n, L, dt, H = 2048, 32.0, 0.02, 0.1
    pp = _uniform(n, L, 31)
    pm = _uniform(n, L, 32)
    rng = np.random.default_rng(3)
    vp = (rng.standard_normal((n, 3)) * 0.5).astype(np.float32)
    vm = (rng.standard_normal((n, 3)) * 0.5).astype(np.float32)
    s = J.Solver(J.Config(box_L=L, pm_grid=32, mu=2.0, G_mass_plus=1e-2, mode=J.JT_ACCURATE))
    s.set_state(pp, vp, pm, vm)
    a0p, a0m = s.accel()
    half = lambda v, a: v + (a - H * v) * (dt / 2)
    wrap = lambda x: np.where(x > L / 2, x - L, np.where(x < -L / 2, x + L, x))
    v1p, v1m = half(vp, a0p), half(vm, a0m)
    x1p, x1m = wrap(pp + v1p * dt), wrap(pm + v1m * dt)
    s.step(dt, H, 1.0, 1)
    gp, gvp, gm, gvm = s.get_state()
    assert np.abs(gp - x1p).max() < 1e-4
    s2 = J.Solver(J.Config(box_L=L, pm_grid=32, mu=2.0, G_mass_plus=1e-2, mode=J.JT_ACCURATE))
    s2.set_state(x1p, None, x1m, None)
    a1p, a1m = s2.accel()
    assert np.abs(gvp - half(v1p, a1p)).max() < 1e-4 * max(1.0, np.abs(gvp).max())
    assert np.abs(gvm - half(v1m, a1m)).max() < 1e-4 * max(1.0, np.abs(gvm).max())
    s.close()
    s2.close()


def test_twopass_mirror_energy_screening_and_segregation():
    """The GpuNBodyTwoPass mirror's energy, virialization, segregation and
    screening methods against the oracle / Solver on the same signed array."""
    J, O = _mods()
    L, n = 40.0, 3000
    rng = np.random.default_rng(23)
    pos = _uniform(n, L, 9)
    vel = rng.normal(0, 0.2, (n, 3)).astype(np.float32)
    sg = np.where(rng.random(n) < 0.5, 1, -1).astype(np.int8)
    sim = J.GpuNBodyTwoPass.with_custom_ics(pos, vel, sg, L, pm_grid=32)
    sim.set_softening(0.05)
    ke = sim.kinetic_energy()
    assert ke == pytest.approx(0.5 * float(np.sum(vel.astype(np.float64) ** 2)), rel=1e-10)
    pe = sim.potential_energy_binding_sampled(1000)
    pe_p, pe_m = O.pe_binding_sampled(pos[sg > 0], pos[sg < 0], 1000, 0.05)
    assert pe == pytest.approx(pe_p + pe_m, rel=1e-10)
    assert sim.segregation() == pytest.approx(O.segregation(pos, sg, L), rel=1e-9, abs=1e-15)
    sim.set_lambda_0(1.93)
    sim.set_current_z(0.8)
    a = sim.compute_forces(5.0)
    ref = O.ref_total_forces_screened(pos, sg, 32, L, 0.5, 0.05, 5.0, sim.mass_factor, 1.93, 0.8)
    rel = _rel(a, ref)
    assert np.percentile(rel, 99) <= 1e-5
    alpha = sim.virialize_sampled(1000)
    _, v2, _ = sim.get_particles()
    assert np.allclose(v2, vel * np.float32(alpha), rtol=1e-6, atol=0)


@pytest.mark.parametrize("k_min", [2, 3])
def test_kmin_filter_both_modes(k_min):
    """The k_min filter (cuda/cufft_wrapper.cu:196-203: modes with
    max(|kx|, |ky|, |kz|) < k_min zeroed) on the device, in both modes, on the
    long-range part alone (JT_PART_PM): compatibility mode against the
    restatement of the reference's PM (p99 <= 1e-5), accurate mode against
    the FP64 PM of the same scheme (PCS, interlaced; p99 <= 1e-4 of the
    unfiltered force's rms).  The filter must also change the force: without
    it the result differs."""
    J, O = _mods()
    L, M, n = 48.0, 32, 3000
    pos = _uniform(n, L, 41)
    rng = np.random.default_rng(42)
    sg = np.where(rng.random(n) < 0.5, 1, -1).astype(np.int8)
    theta, eps, r_cut, mf = 0.5, 0.05, 4.5 * 1.25 * L / M, 0.01
    # compatibility mode: the reference's Green's function with the filter
    s = J.Solver(J.Config(box_L=L, pm_grid=M, theta=theta, softening=eps, r_s=r_cut / 3, r_cut=r_cut,
                          mu=(sg < 0).sum() / (sg > 0).sum(), G_mass_plus=mf, k_min=k_min,
                          mode=J.JT_RCOMPAT))
    pp, pm = pos[sg > 0], pos[sg < 0]
    s.set_state(pp, None, pm, None)
    got = np.concatenate(s.accel_part(J.JT_PART_PM))
    s.close()
    # the per-species layout is the array [m+ ; m-] with its signs
    cat = np.concatenate([pp, pm])
    csg = np.concatenate([np.ones(len(pp), np.int8), -np.ones(len(pm), np.int8)])
    ref = O.ref_pm_forces(cat, csg, M, L, mf, r_cut, k_min=k_min)
    unf = O.ref_pm_forces(cat, csg, M, L, mf, r_cut, k_min=0)
    rel = _rel(got, ref)
    assert np.percentile(rel, 99) <= 1e-5, np.percentile(rel, [50, 99, 100])
    assert np.percentile(_rel(unf, ref), 50) > 1e-3   # the filter changes the force
    # accurate mode: FP64 PM of the same scheme with the same filter
    r_s = 1.25 * L / M
    mass = np.concatenate([np.full(len(pp), 1.0), np.full(len(pm), 19.0 * len(pp) / len(pm))])
    s = J.Solver(J.Config(box_L=L, pm_grid=M, theta=theta, softening=eps, r_s=r_s, r_cut=4.5 * r_s,
                          mu=19.0, G_mass_plus=1.0, k_min=k_min, mode=J.JT_ACCURATE))
    s.set_state(pp, None, pm, None)
    a = np.concatenate(s.accel_part(J.JT_PART_PM)).astype(np.float64)
    s.close()
    p64 = np.concatenate([pp, pm]).astype(np.float64)
    s64 = np.concatenate([np.ones(len(pp), np.int8), -np.ones(len(pm), np.int8)])
    ex = O.acc_pm_forces(p64, mass, s64, M, L, r_s, k_min=k_min, order=4, interlace=True)
    ex0 = O.acc_pm_forces(p64, mass, s64, M, L, r_s, k_min=0, order=4, interlace=True)
    rms = np.sqrt(np.mean(np.sum(ex0 ** 2, axis=1)))
    d = np.linalg.norm(a - ex, axis=1) / rms
    assert np.percentile(d, 99) <= 1e-4, np.percentile(d, [50, 99, 100])
    assert np.percentile(np.linalg.norm(ex0 - ex, axis=1) / rms, 50) > 1e-3
