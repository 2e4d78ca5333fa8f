"""Batched ensembles on the GPU: each box's result is the same alone and in
the mix.

A jt_batch runs every stage as one launch over the work of all its boxes
(uneven particle counts, box sizes, grids, mu, steps).  A box stepped alone
through a single handle and the same box stepped inside a batch of uneven
boxes run the same kernels on the same inputs; the only differences come from
the order of floating-point atomics in the deposit (PM force, ~1e-7
relative).  Tolerances: forces max |a_batch - a_alone| <= 2e-5 x
rms|a_alone|; after 3 KDK steps positions and velocities within 1e-6 x L and
1e-4 x rms|v| (a particle whose Morton key flips on a last-bit position
difference sees a different tree, which stays far inside these bounds over
three steps).
"""
import numpy as np
import pytest

import janus_treepm as J

pytestmark = pytest.mark.gpu

FORCE_TOL = 2e-5
POS_TOL_L = 1e-6
VEL_TOL = 1e-4


def make_box(seed, n_side_p, n_side_m, L, M, mu, theta=0.5):
    rng = np.random.default_rng(seed)
    n_p, n_m = n_side_p ** 3, n_side_m ** 3
    pp = rng.uniform(-L / 2, L / 2, (n_p, 3)).astype(np.float32)
    pm = rng.uniform(-L / 2, L / 2, (n_m, 3)).astype(np.float32)
    vp = rng.normal(0, 0.5, (n_p, 3)).astype(np.float32)
    vm = rng.normal(0, 0.5, (n_m, 3)).astype(np.float32)
    spacing = L / max(n_p + n_m, 1) ** (1 / 3)
    cfg = J.Config(box_L=L, pm_grid=M, theta=theta, softening=spacing / 30, mu=mu,
                   G_mass_plus=1e-3 * (L / 64.0) ** 3)
    return cfg, pp, vp, pm, vm


BOXES = [
    # seed, n+ side, n- side, L, M, mu
    (1, 16, 16, 64.0, 32, 19.0),
    (2, 20, 12, 120.0, 64, 5.0),
    (3, 9, 24, 50.0, 64, 30.0),
    (4, 24, 24, 300.0, 64, 11.0),
    (5, 12, 0, 80.0, 32, 19.0),       # no m- particles
    (6, 1, 2, 40.0, 32, 3.0),         # tiny box: 1 m+, 8 m-
    (7, 30, 30, 200.0, 128, 7.0),
]


def _alone_forces(box):
    cfg, pp, vp, pm, vm = make_box(*box)
    s = J.Solver(cfg)
    s.set_state(pp, vp, pm, vm)
    ap, am = s.accel()
    s.close()
    return ap, am


def _cmp(a, b, tol):
    if len(a) == 0:
        return
    rms = float(np.sqrt(np.mean(np.sum(b.astype(np.float64) ** 2, axis=1))))
    err = float(np.max(np.abs(a.astype(np.float64) - b)))
    assert err <= tol * rms, (err, rms)


def test_pair_counters_leave_the_forces_unchanged():
    """The cell walk's pair counters (a diagnostic, off by default) leave the
    forces as they are, to the rounding of the summation order (neither the
    cell list's order, filled by atomics, nor the deposit's float reductions
    are reproducible bit for bit between runs); with them off the cell walk's
    pairs are not counted (every target of this uniform box takes the cell
    walk)."""
    cfg, pp, vp, pm, vm = make_box(*BOXES[0])
    out = []
    for on in (False, True):
        s = J.Solver(cfg)
        s.set_counters(on)
        s.set_state(pp, vp, pm, vm)
        a = s.accel()
        out.append((a, s.timings()))
        s.close()
    (a0, t0), (a1, t1) = out
    _cmp(a0[0], a1[0].astype(np.float64), 1e-5)
    _cmp(a0[1], a1[1].astype(np.float64), 1e-5)
    assert t1["pair_interactions"] > 0 and t0["pair_interactions"] == 0, (t0, t1)


def test_forces_same_alone_and_in_the_mix():
    B = J.Batch()
    B.set_counters(True)
    ids = []
    for box in BOXES:
        cfg, pp, vp, pm, vm = make_box(*box)
        ids.append(B.add(cfg, pp, vp, pm, vm))
    B.forces(ids)
    t = B.timings()
    # one launch per stage for all seven boxes: 15 (the tiled PM interpolation
    # included), and 6 for the near-field cell list (keys, 3-kernel scan,
    # scatter, cell walk)
    assert t["launches"] == 21
    assert t["pair_interactions"] > 0
    for bid, box in zip(ids, BOXES):
        ap, am = B.accel(bid)
        rp, rm = _alone_forces(box)
        assert np.all(np.isfinite(ap)) and np.all(np.isfinite(am))
        _cmp(ap, rp, FORCE_TOL)
        _cmp(am, rm, FORCE_TOL)
    B.close()


def test_subset_forces_match_full_batch():
    B = J.Batch()
    ids = [B.add(*make_box(*box)) for box in BOXES]
    B.forces(ids)
    full = {i: B.accel(i) for i in ids}
    sub = ids[1::2]
    B.forces(sub)
    for i in sub:
        ap, am = B.accel(i)
        _cmp(ap, full[i][0], FORCE_TOL)
        _cmp(am, full[i][1], FORCE_TOL)
    B.close()


def test_steps_same_alone_and_in_the_mix():
    dts = [0.01, 0.02, 0.005, 0.01, 0.015, 0.01, 0.02]
    hub = [0.0, 0.1, 0.05, 0.2, 0.0, 0.0, 0.07]
    B = J.Batch()
    ids = []
    for box in BOXES:
        cfg, pp, vp, pm, vm = make_box(*box)
        ids.append(B.add(cfg, pp, vp, pm, vm))
    B.step(ids, dts, hub, 1.0, nsteps=3)
    for k, (bid, box) in enumerate(zip(ids, BOXES)):
        cfg, pp, vp, pm, vm = make_box(*box)
        s = J.Solver(cfg)
        s.set_state(pp, vp, pm, vm)
        s.step(dts[k], hub[k], 1.0, 3)
        ref = s.get_state()
        s.close()
        got = B.get_state(bid)
        for q, (g, r) in enumerate(zip(got, ref)):
            if len(r) == 0:
                continue
            d = np.abs(g.astype(np.float64) - r)
            if q % 2 == 0:                                # positions (periodic)
                d = np.minimum(d, cfg.box_L - d)
                assert float(d.max()) <= POS_TOL_L * cfg.box_L, (k, q, float(d.max()))
            else:
                rms = float(np.sqrt(np.mean(np.sum(r.astype(np.float64) ** 2, axis=1))))
                assert float(d.max()) <= VEL_TOL * rms, (k, q, float(d.max()), rms)
    B.close()


def test_remove_and_reuse_slot():
    B = J.Batch()
    a = B.add(*make_box(*BOXES[0]))
    b = B.add(*make_box(*BOXES[1]))
    B.forces([a, b])
    ref_b = B.accel(b)
    B.remove(a)
    c = B.add(*make_box(*BOXES[3]))
    assert c == a                      # freed id reused
    B.forces([b, c])
    got_b = B.accel(b)
    _cmp(got_b[0], ref_b[0], FORCE_TOL)
    _cmp(got_b[1], ref_b[1], FORCE_TOL)
    pers, scratch = B.memory()
    est = sum(sum(J.Batch.estimate(make_box(*BOXES[i])[0], BOXES[i][1] ** 3, BOXES[i][2] ** 3))
              for i in (1, 3))
    assert pers > 0 and scratch > 0 and est > 0
    B.close()


def test_batch_rejects_mismatched_shared_fields():
    B = J.Batch()
    B.add(*make_box(*BOXES[0]))
    cfg, pp, vp, pm, vm = make_box(*BOXES[1])
    cfg.pm_interlace = 2               # the batch's boxes are interlaced
    with pytest.raises(J.JanusError) as e:
        B.add(cfg, pp, vp, pm, vm)
    assert e.value.code == J.JT_EINVAL
    with pytest.raises(J.JanusError):
        B.forces([0, 0])               # duplicate id
    with pytest.raises(J.JanusError):
        B.forces([5])                  # unknown id
    B.close()


def test_graph_replay_matches_plain_launches():
    dts = [0.01, 0.02, 0.005, 0.01, 0.015, 0.01, 0.02]
    hub = [0.0, 0.1, 0.05, 0.2, 0.0, 0.0, 0.07]
    A, G = J.Batch(), J.Batch(graphs=True)
    ia = [A.add(*make_box(*box)) for box in BOXES]
    ig = [G.add(*make_box(*box)) for box in BOXES]
    # odd and even step counts (both graph parities), a dt change between
    # calls, and a subset (a second capture) in between
    for n, scale in ((3, 1.0), (2, 0.5)):
        A.step(ia, [d * scale for d in dts], hub, 1.0, nsteps=n)
        G.step(ig, [d * scale for d in dts], hub, 1.0, nsteps=n)
        A.step(ia[:3], dts[:3], hub[:3], 1.0, nsteps=1)
        G.step(ig[:3], dts[:3], hub[:3], 1.0, nsteps=1)
    assert G.timings()["launches"] > 0
    for k, box in enumerate(BOXES):
        L = make_box(*box)[0].box_L
        for q, (g, r) in enumerate(zip(G.get_state(ig[k]), A.get_state(ia[k]))):
            if len(r) == 0:
                continue
            d = np.abs(g.astype(np.float64) - r)
            if q % 2 == 0:
                d = np.minimum(d, L - d)
                assert float(d.max()) <= POS_TOL_L * L, (k, q, float(d.max()))
            else:
                rms = float(np.sqrt(np.mean(np.sum(r.astype(np.float64) ** 2, axis=1))))
                assert float(d.max()) <= VEL_TOL * rms, (k, q, float(d.max()), rms)
    A.close()
    G.close()


def test_async_checkpoint_overlaps_the_next_step(tmp_path):
    """A checkpoint started before a step holds the state before it, and the
    step's result is the same as without the checkpoint."""
    import janus_treepm as J
    rng = np.random.default_rng(21)
    L, n = 50.0, 6000
    cfg = J.Config(box_L=L, pm_grid=32, softening=0.05, mu=3.0)
    st = []
    for _ in range(2):
        st.append([((rng.random((n, 3)) - 0.5) * L).astype(np.float32), rng.normal(0, 0.3, (n, 3)).astype(np.float32),
                   ((rng.random((n // 2, 3)) - 0.5) * L).astype(np.float32),
                   rng.normal(0, 0.3, (n // 2, 3)).astype(np.float32)])
    B = J.Batch()
    ids = [B.add(cfg, *s) for s in st]
    B.step(ids, 0.01, 0.0, 1.0, 2)
    before = B.get_state(ids[0])
    path = tmp_path / "ck.bin"
    B.checkpoint_async(ids[0], path, J.snapshot_meta(run_label="async"))
    B.step(ids, 0.01, 0.0, 1.0, 1)
    B.checkpoint_wait()
    after = B.get_state(ids[0])
    meta, L2, mu2, pos, vel, sg, mass, eps = J.snapshot_read(path)
    assert meta.run_label == b"async" and L2 == L and mu2 == 3.0
    assert np.array_equal(pos, np.concatenate([before[0], before[2]]))
    assert np.array_equal(vel, np.concatenate([before[1], before[3]]))
    assert np.array_equal(sg, np.concatenate([np.ones(n, np.int8), -np.ones(n // 2, np.int8)]))
    # the same step from the saved state without a checkpoint in flight
    B2 = J.Batch()
    i2 = [B2.add(cfg, *s) for s in st]
    B2.step(i2, 0.01, 0.0, 1.0, 2)
    B2.step(i2, 0.01, 0.0, 1.0, 1)
    ref = B2.get_state(i2[0])
    for x, y in zip(after, ref):
        assert np.abs(x - y).max() <= 1e-5 * max(1.0, np.abs(y).max())
    B.close()
    B2.close()


def test_cell_walk_matches_the_tree_walk():
    """The near-field cell walk against the tree walk alone (JT_WALK_CELLS=0)
    on uniform boxes at theta = 0.1, where the tree accepts no multipole
    inside r_cut: the same pairs, in another order (forces p99 within 2e-5
    of rms), and the same pair count to a few borderline pairs at r_cut.  A box
    with fewer than 3 cells per axis takes the tree walk either way."""
    import os
    out = {}
    for cells in ("1", "0"):
        os.environ["JT_WALK_CELLS"] = cells
        try:
            B = J.Batch()
            B.set_counters(True)
            ids = []
            # the third box: r_cut = 8 in L = 20, 2 cells per axis
            for k, (L, M, n, rc) in enumerate(((60.0, 32, 20, 0.0), (40.0, 64, 16, 0.0), (20.0, 16, 8, 8.0))):
                rng = np.random.default_rng(70 + k)
                pp = rng.uniform(-L / 2, L / 2, (n ** 3, 3)).astype(np.float32)
                pm = rng.uniform(-L / 2, L / 2, (n ** 3, 3)).astype(np.float32)
                cfg = J.Config(box_L=L, pm_grid=M, theta=0.1, softening=0.02 * L / n, mu=3.0,
                               G_mass_plus=1e-3, r_cut=rc)
                ids.append(B.add(cfg, pp, None, pm, None))
            B.forces(ids)
            out[cells] = ([B.accel(i) for i in ids], B.timings())
            B.close()
        finally:
            os.environ.pop("JT_WALK_CELLS", None)
    # a pair right at r_cut can fall on either side of the cut between the
    # two paths' rounding (S(2.25) = 1.8 % of its Newtonian force), and the
    # deposit's atomics differ in order: p99 and max bars, not max alone
    for (ap, am), (bp, bm) in zip(out["1"][0], out["0"][0]):
        for a, b in ((ap, bp), (am, bm)):
            rms = float(np.sqrt(np.mean(np.sum(b.astype(np.float64) ** 2, axis=1))))
            d = np.linalg.norm(a.astype(np.float64) - b, axis=1) / rms
            assert np.percentile(d, 99) <= 2e-5 and d.max() <= 2e-3, (np.percentile(d, 99), d.max())
    p1, p0 = out["1"][1]["pair_interactions"], out["0"][1]["pair_interactions"]
    assert abs(p1 - p0) <= 1e-4 * p0, (p1, p0)
    # with the cells off the cell-walk events are recorded back to back
    assert out["1"][1]["cellwalk_ms"] > 0.0 and out["0"][1]["cellwalk_ms"] < 0.01


SCREEN = {0: (5.0, 0.0), 2: (3.0, 1.0), 3: (40.0, 0.5)}   # box index -> (lambda_0, z)


def test_screened_boxes_same_alone_and_in_the_mix():
    """Screened and unscreened boxes in one batch: each box's forces equal
    its own single-box result, and the pass adds one launch (the unsigned
    source's deposit).  Graph replay of screened steps matches plain
    launches; turning screening off restores the unscreened forces."""
    boxes = BOXES[:5]
    B = J.Batch()
    ids = [B.add(*make_box(*box)) for box in boxes]
    for k, (lam, z) in SCREEN.items():
        B.set_screening(ids[k], lam, z)
    B.forces(ids)
    assert B.timings()["launches"] == 21
    for k, (bid, box) in enumerate(zip(ids, boxes)):
        cfg, pp, vp, pm, vm = make_box(*box)
        s = J.Solver(cfg)
        if k in SCREEN:
            s.set_screening(*SCREEN[k])
        s.set_state(pp, vp, pm, vm)
        rp, rm = s.accel()
        s.close()
        ap, am = B.accel(bid)
        _cmp(ap, rp, FORCE_TOL)
        _cmp(am, rm, FORCE_TOL)
        if k in SCREEN:   # screening is visible at this scale
            ref = _alone_forces(box)
            assert np.abs(ap.astype(np.float64) - ref[0]).max() > 100 * FORCE_TOL * np.abs(ref[0]).max()
    for k in SCREEN:
        B.set_screening(ids[k], 0.0)
    B.forces(ids)
    for k, (bid, box) in enumerate(zip(ids, boxes)):
        ap, am = B.accel(bid)
        rp, rm = _alone_forces(box)
        _cmp(ap, rp, FORCE_TOL)
        _cmp(am, rm, FORCE_TOL)
    B.close()

    dts = [0.01, 0.02, 0.005, 0.01, 0.015]
    hub = [0.0, 0.1, 0.05, 0.2, 0.0]
    A, G = J.Batch(), J.Batch(graphs=True)
    ia = [A.add(*make_box(*box)) for box in boxes]
    ig = [G.add(*make_box(*box)) for box in boxes]
    for k, (lam, z) in SCREEN.items():
        A.set_screening(ia[k], lam, z)
        G.set_screening(ig[k], lam, z)
    A.step(ia, dts, hub, 1.0, nsteps=3)
    G.step(ig, dts, hub, 1.0, nsteps=3)
    for k, box in enumerate(boxes):
        L = make_box(*box)[0].box_L
        for q, (g, r) in enumerate(zip(G.get_state(ig[k]), A.get_state(ia[k]))):
            if len(r) == 0:
                continue
            d = np.abs(g.astype(np.float64) - r)
            if q % 2 == 0:
                d = np.minimum(d, L - d)
                assert float(d.max()) <= POS_TOL_L * L, (k, q, float(d.max()))
            else:
                rms = float(np.sqrt(np.mean(np.sum(r.astype(np.float64) ** 2, axis=1))))
                assert float(d.max()) <= VEL_TOL * rms, (k, q, float(d.max()), rms)
    A.close()
    G.close()


def test_prepared_plans_change_nothing():
    """jt_batch_prepare makes the cuFFT plans of a grid size ahead: the same
    forces as a batch that makes them in its first pass; sizes that are not
    powers of two in [8, 1024] are refused."""
    boxes = BOXES[:3]
    A, P = J.Batch(), J.Batch()
    for M in sorted({b[4] for b in boxes}):
        P.prepare(M)
    with pytest.raises(J.JanusError):
        P.prepare(48)
    ia = [A.add(*make_box(*box)) for box in boxes]
    ip = [P.add(*make_box(*box)) for box in boxes]
    A.forces(ia)
    P.forces(ip)
    for a, p in zip(ia, ip):
        for x, y in zip(P.accel(p), A.accel(a)):
            _cmp(x, y, FORCE_TOL)
    A.close()
    P.close()


def test_cell_count_autotuner_single_species():
    """A box of 2^22 particles (one species) takes the cell-count autotuner on
    its first force pass: the forces agree with the default cell count's to
    the rounding of the summation order, and jt_walk_tuning reports the box.
    The default run is a child process (JT_CELL_TUNE=0 is read once)."""
    import json
    import os
    import subprocess
    import sys
    n, L, M = 1 << 22, 160.0, 256
    code = f"""
import sys, numpy as np
sys.path.insert(0, {os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), 'janus-sim_b200')!r})
import janus_treepm as J
rng = np.random.default_rng(5)
pp = rng.uniform(-{L} / 2, {L} / 2, ({n}, 3)).astype(np.float32)
cfg = J.Config(box_L={L}, pm_grid={M}, theta=0.5, softening=0.02, mu=19.0, G_mass_plus=1e-3,
               mode=J.JT_ACCURATE, cut_tail_ppm=440)
s = J.Solver(cfg)
s.set_state(pp, None, np.zeros((0, 3), np.float32), None)
ap, _ = s.accel_part(J.JT_PART_SHORT)
np.save(sys.argv[1], ap)
print(J.walk_tuning())
"""
    import tempfile
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for tune in ("1", "0"):
            f = os.path.join(tmp, f"a{tune}.npy")
            env = dict(os.environ, JT_CELL_TUNE=tune)
            r = subprocess.run([sys.executable, "-c", code, f], env=env, capture_output=True, text=True,
                               timeout=600)
            assert r.returncode == 0, r.stderr[-2000:]
            out[tune] = (np.load(f), r.stdout)
    a1, a0 = out["1"][0].astype(np.float64), out["0"][0].astype(np.float64)
    rms = float(np.sqrt(np.mean(np.sum(a0 ** 2, axis=1))))
    assert np.all(np.isfinite(a1)) and float(np.abs(a1 - a0).max()) <= 1e-4 * rms
    assert f"cells {n} particles:" in out["1"][1]
    assert f"cells {n} particles:" not in out["0"][1]
