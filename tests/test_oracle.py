"""The oracle, pinned (CPU only).

1. Against the golden fixtures in tests/golden/ (made by make_golden.py from
   the reference's own kernels compiled for the host): the restatements must
   reproduce them exactly (integer arrays) or bit-for-bit (float arrays; both
   are evaluated without fused multiply-adds on the same CPU).
2. Against the reference kernels live (oracle/_ref), when that harness is
   built here, on fresh seeded inputs.
3. The reference's own qualitative tests for this path (src/treepm/*.rs
   #[cfg(test)], tests/treepm_physics_8p.rs, tests/treepm_isotropy.rs):
   sign rules, symmetry, CIC mass conservation, isotropy.
4. The FP64 Ewald oracle against closed forms.
"""
import os

import numpy as np
import pytest

import oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return dict(np.load(os.path.join(GOLD, name)))


# ---------------------------------------------------------------- 1. golden
@pytest.mark.parametrize("name", ["tree_uniform_2000.npz", "tree_collide_1500.npz"])
def test_tree_matches_golden(name):
    g = load(name)
    pos, bh, mass = g["pos"], g["box_half"], g["mass"]
    T = O.build_tree(pos, bh, mass)
    m30 = (g["keys"] >> np.uint64(32)).astype(np.uint32)
    assert np.array_equal(T["m30"], m30)
    assert np.array_equal(T["perm"], g["perm"])
    assert np.array_equal(T["left"][:len(pos) - 1], g["left"])
    assert np.array_equal(T["right"][:len(pos) - 1], g["right"])
    assert np.array_equal(T["parent"], g["parent"])
    assert np.array_equal(T["rl"], g["rl"])
    assert np.array_equal(T["rr"], g["rr"])
    assert np.array_equal(T["node_pos"], g["node_pos"])
    assert np.array_equal(T["node_mass"], g["node_mass"])
    assert np.array_equal(T["types"], g["types"])


def test_collision_fixture_has_ties():
    g = load("tree_collide_1500.npz")
    m30 = (g["keys"] >> np.uint64(32)).astype(np.uint32)
    assert len(np.unique(m30)) < len(m30) // 2


def test_pm_matches_golden():
    g = load("forces_mixed_1200.npz")
    pos, sg, M, L = g["pos"], g["signs"], int(g["M"]), float(g["L"])
    G = M ** 3
    rp, rm = np.zeros(G), np.zeros(G)
    bh, ic, cell = np.float32(L / 2), np.float32(M / L), np.float32(L / M)
    O.lib().orc_ref_cic_scatter(pos.ravel(), sg, len(pos), M, bh, ic, rp, rm)
    assert np.array_equal(rp, g["rho_plus"]) and np.array_equal(rm, g["rho_minus"])
    g_const = float(g["mass_factor"]) / (L / M) ** 3
    pp, pm = np.zeros(G), np.zeros(G)
    O.lib().orc_ref_poisson(rp, pp, M, L, g_const, float(g["r_cut"]) / 3.0, 0)
    O.lib().orc_ref_poisson(rm, pm, M, L, g_const, float(g["r_cut"]) / 3.0, 0)
    scale = np.abs(g["phi_plus"]).max()
    assert np.abs(pp - g["phi_plus"]).max() <= 1e-12 * scale
    assert np.abs(pm - g["phi_minus"]).max() <= 1e-12 * scale
    f = np.zeros(3 * len(pos), np.float32)
    O.lib().orc_ref_cic_gather(pos.ravel(), sg, len(pos), M, bh, ic, cell, g["phi_plus"],
                               g["phi_minus"], f)
    assert np.array_equal(f.reshape(-1, 3), g["pm_forces"])


def test_kmin_filter_matches_golden():
    g = load("pm_kmin3_1200.npz")
    pos, sg, M, L = g["pos"], g["signs"], int(g["M"]), float(g["L"])
    G = M ** 3
    rp, rm = np.zeros(G), np.zeros(G)
    O.lib().orc_ref_cic_scatter(pos.ravel(), sg, len(pos), M, np.float32(L / 2),
                                np.float32(M / L), rp, rm)
    pp = np.zeros(G)
    O.lib().orc_ref_poisson(rp, pp, M, L, float(g["g_const"]), float(g["r_s"]), 3)
    assert np.abs(pp - g["phi_plus"]).max() <= 1e-12 * np.abs(g["phi_plus"]).max()


def test_short_range_walk_matches_golden():
    g = load("forces_mixed_1200.npz")
    pos, sg, L = g["pos"], g["signs"], float(g["L"])
    tq, sq, rq, bq = O.ref_quantize(float(g["theta"]), float(g["eps"]), float(g["r_cut"]), L)
    acc = np.zeros(3 * len(pos), np.float32)
    for k, s in enumerate((1, -1)):
        T = O.build_tree(np.ascontiguousarray(pos[sg == s]), np.float32(L / 2), float(g["mass_factor"]))
        O.lib().orc_ref_short_range(pos.ravel(), sg, len(pos), s, T["node_pos"].ravel(),
                                    T["node_mass"], T["left"], T["right"], T["types"],
                                    tq, sq, rq, bq, k, acc)
    assert np.array_equal(acc.reshape(-1, 3), g["short"])


def test_total_reference_force_matches_golden():
    g = load("forces_mixed_1200.npz")
    acc = O.ref_total_forces(g["pos"], g["signs"], int(g["M"]), float(g["L"]), float(g["theta"]),
                             float(g["eps"]), float(g["r_cut"]), float(g["mass_factor"]))
    rel = np.linalg.norm(acc - g["total"], axis=1) / np.linalg.norm(g["total"], axis=1)
    assert rel.max() < 1e-5   # f64 FFT implementations differ in the last bits only


def test_screened_walk_matches_golden():
    g = load("screened_mixed_1100.npz")
    pos, sg, L = g["pos"], g["signs"], float(g["L"])
    tq, sq, il, bq = O.ref_screen_quantize(float(g["theta"]), float(g["eps"]), float(g["lambda_0"]),
                                           float(g["z"]), L)
    # rounding (screened packing) and truncation (erfc-split packing) differ here
    assert (tq, sq) != O.ref_quantize(float(g["theta"]), float(g["eps"]), 5.0, L)[:2]
    acc = np.zeros(3 * len(pos), np.float32)
    for k, s in enumerate((1, -1)):
        T = O.build_tree(np.ascontiguousarray(pos[sg == s]), np.float32(L / 2), float(g["mass_factor"]))
        O.lib().orc_ref_screened_walk(pos.ravel(), sg, len(pos), s, T["node_pos"].ravel(),
                                      T["node_mass"], T["left"], T["right"], T["types"],
                                      tq, sq, il, bq, k, acc)
    assert np.array_equal(acc.reshape(-1, 3), g["screened"])
    tot = O.ref_total_forces_screened(pos, sg, int(g["M"]), L, float(g["theta"]), float(g["eps"]),
                                      float(g["r_cut"]), float(g["mass_factor"]),
                                      float(g["lambda_0"]), float(g["z"]))
    rel = np.linalg.norm(tot - g["total"], axis=1) / np.linalg.norm(g["total"], axis=1)
    assert rel.max() < 1e-5   # f64 FFT implementations differ in the last bits only


def test_screening_limits():
    """lambda_0 <= 0.01 is the unscreened erfc-split path; a huge lambda makes
    the screening factor 1 (the plain full-range walk); tiny 1/lambda removes
    nothing from same-sign pairs."""
    rng = np.random.default_rng(2)
    n, L = 600, 30.0
    pos = ((rng.random((n, 3)) - 0.5) * L).astype(np.float32)
    sg = np.where(rng.random(n) < 0.5, 1, -1).astype(np.int8)
    a0 = O.ref_total_forces(pos, sg, 16, L, 0.5, 0.05, 5.0, 0.02)
    a1 = O.ref_total_forces_screened(pos, sg, 16, L, 0.5, 0.05, 5.0, 0.02, 0.005, 0.0)
    assert np.array_equal(a0, a1)
    _, _, il, _ = O.ref_screen_quantize(0.5, 0.05, 6000.0, 0.0, L)
    assert 0 < il < 2e-4
    # screening weakens only the opposite-sign (repulsive) part: with all
    # particles of one sign the result does not depend on lambda
    one = np.ones(n, np.int8)
    b1 = O.ref_total_forces_screened(pos, one, 16, L, 0.5, 0.05, 5.0, 0.02, 0.5, 0.0)
    b2 = O.ref_total_forces_screened(pos, one, 16, L, 0.5, 0.05, 5.0, 0.02, 50.0, 3.0)
    assert np.array_equal(b1, b2)


# ---------------------------------------------------------------- 2. live reference
needs_ref = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")


@needs_ref
@pytest.mark.parametrize("seed,n", [(1, 3000), (2, 777), (3, 2)])
def test_tree_matches_reference_kernels_live(seed, n):
    import sys
    sys.path.insert(0, GOLD)
    from make_golden import ref_tree
    rng = np.random.default_rng(seed)
    pos = ((rng.random((n, 3)) - 0.5) * 100.0).astype(np.float32)
    pos[: n // 3] = pos[n // 3: 2 * (n // 3)]  # exact duplicates too
    g = ref_tree(pos, 50.0, 0.5)
    T = O.build_tree(pos, np.float32(50.0), 0.5)
    assert np.array_equal(T["perm"], g["perm"])
    assert np.array_equal(T["left"][:n - 1], g["left"])
    assert np.array_equal(T["right"][:n - 1], g["right"])
    assert np.array_equal(T["parent"], g["parent"])
    assert np.array_equal(T["node_pos"], g["node_pos"])


@needs_ref
def test_walk_matches_reference_kernel_live():
    import sys
    sys.path.insert(0, GOLD)
    from make_golden import ref_short, ref_tree
    rng = np.random.default_rng(9)
    n, L = 900, 40.0
    pos = ((rng.random((n, 3)) - 0.5) * L).astype(np.float32)
    sg = np.where(rng.random(n) < 0.5, 1, -1).astype(np.int8)
    theta, eps, r_cut, mf = 0.6, 0.03, 4.2, 0.1
    trees = [ref_tree(np.ascontiguousarray(pos[sg == s]), L / 2, mf) for s in (1, -1)]
    a_ref = ref_short(pos, sg, trees, theta, eps, r_cut, L)
    tq, sq, rq, bq = O.ref_quantize(theta, eps, r_cut, L)
    acc = np.zeros(3 * n, np.float32)
    for k, s in enumerate((1, -1)):
        T = O.build_tree(np.ascontiguousarray(pos[sg == s]), np.float32(L / 2), mf)
        O.lib().orc_ref_short_range(pos.ravel(), sg, n, s, T["node_pos"].ravel(), T["node_mass"],
                                    T["left"], T["right"], T["types"], tq, sq, rq, bq, k, acc)
    assert np.array_equal(acc.reshape(-1, 3), a_ref)


@needs_ref
@pytest.mark.parametrize("theta,eps,lam,z", [(0.6, 0.0305, 2.37, 1.5), (0.45, 0.1, 0.3, 0.0),
                                            (0.7, 0.02, 6000.0, 9.0)])
def test_screened_walk_matches_reference_kernel_live(theta, eps, lam, z):
    import sys
    sys.path.insert(0, GOLD)
    from make_golden import ref_screened, ref_tree
    rng = np.random.default_rng(13)
    n, L, mf = 1000, 40.0, 0.1
    pos = ((rng.random((n, 3)) - 0.5) * L).astype(np.float32)
    sg = np.where(rng.random(n) < 0.5, 1, -1).astype(np.int8)
    trees = [ref_tree(np.ascontiguousarray(pos[sg == s]), L / 2, mf) for s in (1, -1)]
    a_ref = ref_screened(pos, sg, trees, theta, eps, lam, z, L)
    tq, sq, il, bq = O.ref_screen_quantize(theta, eps, lam, z, L)
    acc = np.zeros(3 * n, np.float32)
    for k, s in enumerate((1, -1)):
        T = O.build_tree(np.ascontiguousarray(pos[sg == s]), np.float32(L / 2), mf)
        O.lib().orc_ref_screened_walk(pos.ravel(), sg, n, s, T["node_pos"].ravel(), T["node_mass"],
                                      T["left"], T["right"], T["types"], tq, sq, il, bq, k, acc)
    assert np.array_equal(acc.reshape(-1, 3), a_ref)


# ---------------------------------------------------------------- 3. reference's own tests
def _cpu_force(pos, signs, mass, r_cut, grid, box, theta=0.5, eps=0.5):
    acc, _, _ = O.cpu_treepm_forces(np.asarray(pos, float), np.asarray(mass, float),
                                    np.asarray(signs, np.int8), r_cut, grid, box, theta, eps)
    return acc


@pytest.mark.parametrize("si,sj,attract", [(1, 1, True), (-1, -1, True), (1, -1, False), (-1, 1, False)])
def test_cpu_treepm_pair_signs(si, sj, attract):
    # treepm_force.rs test_treepm_all_four_signs: particles at x = -10, +10
    acc = _cpu_force([[-10, 0, 0], [10, 0, 0]], [si, sj], [1, 1], 30.0, 32, 100.0)
    assert (acc[0, 0] > 0) == attract


def test_cpu_treepm_symmetry():
    # treepm_force.rs test_treepm_basic: forces on the pair are opposite within 1%
    acc = _cpu_force([[-10, 0, 0], [10, 0, 0]], [1, 1], [1, 1], 20.0, 32, 100.0)
    assert acc[0, 0] > 0 > acc[1, 0]
    assert abs(acc[0, 0] + acc[1, 0]) < 0.01 * abs(acc[0, 0])


def test_ref_cic_mass_conservation():
    # pm_grid.rs test_mass_assignment: CIC of one particle sums to 1
    M = 32
    rp, rm = np.zeros(M ** 3), np.zeros(M ** 3)
    O.lib().orc_ref_cic_scatter(np.array([0.3, -1.7, 2.2], np.float32), np.array([1], np.int8), 1,
                                M, np.float32(50), np.float32(M / 100.0), rp, rm)
    assert abs(rp.sum() - 1.0) < 1e-6 and rm.sum() == 0.0


def test_ref_pm_isotropy():
    # treepm_isotropy.rs: a shell of test particles around a central mass feels
    # forces within 5 degrees of radial (64^3, box 200, shell r = 30)
    M, L = 64, 200.0
    n = 100
    phi_g = np.pi * (3 - np.sqrt(5))
    i = np.arange(n)
    y = 1 - i / (n - 1) * 2
    r = np.sqrt(1 - y * y)
    shell = np.stack([30 * r * np.cos(phi_g * i), 30 * y, 30 * r * np.sin(phi_g * i)], 1)
    pos = np.concatenate([[[0.0, 0.0, 0.0]], shell]).astype(np.float32)
    sg = np.ones(n + 1, np.int8)
    # a test particle of negligible weight: scatter the centre only
    G = M ** 3
    rp, rm = np.zeros(G), np.zeros(G)
    O.lib().orc_ref_cic_scatter(pos[:1].ravel(), sg[:1], 1, M, np.float32(L / 2), np.float32(M / L), rp, rm)
    pp, pm = np.zeros(G), np.zeros(G)
    O.lib().orc_ref_poisson(rp * 100.0, pp, M, L, 1.0, 0.0, 0)
    f = np.zeros(3 * n, np.float32)
    O.lib().orc_ref_cic_gather(pos[1:].ravel(), sg[1:], n, M, np.float32(L / 2), np.float32(M / L),
                               np.float32(L / M), pp, pm, f)
    f = f.reshape(n, 3)
    cosang = np.sum(f * -shell, 1) / (np.linalg.norm(f, axis=1) * 30)
    ang = np.degrees(np.arccos(np.clip(cosang, -1, 1)))
    assert ang.mean() < 5.0 and ang.std() < 5.0


# ---------------------------------------------------------------- 4. Ewald oracle
def test_ewald_pair_newton_third_law_and_sign():
    L = 20.0
    pos = np.array([[-1.0, 0.3, 0.1], [1.5, -0.2, 0.4]])
    mass = np.array([2.0, 3.0])
    for s2 in (1, -1):
        sg = np.array([1, s2], np.int8)
        a = O.ewald_forces(pos, mass, sg, L, 0.8, 0.0)
        f = a * mass[:, None]
        # Janus pairs: m_i a_i = s_i s_j m_i m_j r_ij / r^3 is antisymmetric in
        # (i, j) for both signs -- equal and opposite forces
        assert np.allclose(f[0], -f[1], rtol=1e-9, atol=1e-12)
        if s2 == 1:
            assert a[0, 0] > 0    # attraction: towards the other particle
        else:
            assert a[0, 0] < 0    # repulsion: away from it


def test_ewald_independent_of_split_scale():
    rng = np.random.default_rng(5)
    L = 10.0
    pos = (rng.random((40, 3)) - 0.5) * L
    mass = rng.uniform(0.5, 2.0, 40)
    sg = np.where(rng.random(40) < 0.5, 1, -1).astype(np.int8)
    a1 = O.ewald_forces(pos, mass, sg, L, 0.6, 0.0)
    a2 = O.ewald_forces(pos, mass, sg, L, 1.1, 0.0)
    assert np.abs(a1 - a2).max() < 1e-8 * np.abs(a1).max()


def test_ewald_close_pair_is_newtonian():
    # two particles much closer than the box: force -> 1/r^2 (+ small image terms)
    L = 1000.0
    pos = np.array([[0.0, 0.0, 0.0], [0.5, 0.0, 0.0]])
    a = O.ewald_forces(pos, np.array([1.0, 1.0]), np.array([1, 1], np.int8), L, 5.0, 0.0)
    assert abs(a[0, 0] - 1.0 / 0.25) < 1e-6 * 4.0


@pytest.mark.parametrize("order,interlace,p50_max", [(2, False, 2.5e-2), (2, True, 6e-3),
                                                     (3, False, 4e-3), (3, True, 5e-4),
                                                     (4, False, 3e-3), (4, True, 1e-4)])
def test_acc_pm_against_long_range_ewald(order, interlace, p50_max):
    """PM force errors against the exact long-range (Ewald reciprocal) sum at
    r_s = 1.25 cells: CIC ~1e-2, TSC + interlacing ~2e-4, PCS + interlacing
    ~3e-5 (median)."""
    rng = np.random.default_rng(8)
    L, M, n = 16.0, 32, 300
    pos = (rng.random((n, 3)) - 0.5) * L
    mass = np.ones(n)
    sg = np.where(rng.random(n) < 0.5, 1, -1).astype(np.int8)
    r_s = 1.25 * L / M
    a_pm = O.acc_pm_forces(pos, mass, sg, M, L, r_s, order=order, interlace=interlace)
    a_ex = O.ewald_forces(pos, mass, sg, L, r_s, 0.0, part="long")
    rel = np.linalg.norm(a_pm - a_ex, axis=1) / np.linalg.norm(a_ex, axis=1)
    assert np.median(rel) < p50_max


def test_split_energy_is_the_potential_of_the_oracle_forces():
    """orc_split_energy: independent of r_s for an untruncated split (net
    charge included), and -grad U / m equals orc_ewald_forces on the
    truncated model."""
    L = 20.0
    pos = np.array([[0, 0, 0], [1.5, 0, 0], [3, 4, -2], [-7, 2, 9]], float)
    m = np.array([1.0, 2.0, 0.5, 0.3])
    s = np.array([1, 1, -1, -1], np.int8)
    us = [O.split_energy(pos, m, s, L, rs, 0.0, 12 * rs)[0] for rs in (0.4, 0.6, 0.9)]
    assert max(us) - min(us) <= 1e-10 * abs(us[0])
    rs, eps, h = 0.5, 0.1, 1e-5
    rc = 4.5 * rs
    a = O.ewald_forces(pos, m, s, L, rs, eps, r_trunc=rc)
    for i in range(len(pos)):
        for d in range(3):
            pp, pn = pos.copy(), pos.copy()
            pp[i, d] += h
            pn[i, d] -= h
            g = -(O.split_energy(pp, m, s, L, rs, eps, rc)[0] - O.split_energy(pn, m, s, L, rs, eps, rc)[0]) / (2 * h) / m[i]
            assert abs(g - a[i, d]) <= 1e-6 * max(1.0, abs(a[i, d]))


def test_screened_split_oracle():
    """orc_ewald_forces_screened: kappa = 0 is the unscreened oracle; with
    screening (eps = 0, no truncation) the split sum is independent of r_s;
    two opposite-sign particles in a large box feel exactly
    -m e^{-kappa r}(1 + kappa r) / r^2."""
    rng = np.random.default_rng(3)
    n, L = 60, 10.0
    pos = (rng.random((n, 3)) - 0.5) * L
    m = rng.uniform(0.5, 2.0, n)
    s = np.where(rng.random(n) < 0.5, 1, -1).astype(np.int8)
    a0 = O.ewald_forces(pos, m, s, L, 0.5, 0.1)
    b0 = O.ewald_forces_screened(pos, m, s, L, 0.5, 0.1, 0.0)
    assert np.abs(a0 - b0).max() <= 1e-14 * np.abs(a0).max()
    for kap in (0.3, 1.0, 3.0):
        x = [O.ewald_forces_screened(pos, m, s, L, rs, 0.0, kap) for rs in (0.4, 0.6)]
        assert np.abs(x[0] - x[1]).max() <= 1e-12 * np.abs(x[0]).max()
    pos2 = np.array([[0, 0, 0], [1.3, 0, 0]], float)
    a = O.ewald_forces_screened(pos2, np.array([1.0, 2.0]), np.array([1, -1], np.int8), 40.0, 0.4, 0.0, 1.0)
    assert a[0, 0] == pytest.approx(-2.0 * np.exp(-1.3) * 2.3 / 1.3 ** 2, rel=1e-12)
