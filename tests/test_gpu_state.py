"""State round trips through the host: positions, velocities and the
accelerations a KDK step starts from (jt_get_accel / jt_set_accel).  A
host-driven loop that takes the state out and puts it back every step follows
the device-resident trajectory.  The reload changes the order of equal Morton
keys, hence the 32-particle walk groups and which nodes the opening test
accepts as multipoles.  At theta = 0.1 no node inside r_cut is accepted, so
the two differ only in summation order: positions within 1e-5 L, velocities
within 1e-4 rms after four steps.  The accelerations put back are the ones
read (bit-exact); without forces a reloaded state has none to read
(JT_ESTATE)."""
import numpy as np
import pytest

import janus_treepm as J

pytestmark = pytest.mark.gpu


def test_host_round_trip_follows_the_device_trajectory():
    from janus_treepm import ics
    L, n = 60.0, 20
    pp, vp, pm, vm = ics.zeldovich_lattice(n, L, seed=5)
    cfg = J.Config(box_L=L, pm_grid=32, softening=0.05, mu=3.0, theta=0.1)
    a = J.Solver(cfg)
    a.set_state(pp, vp, pm, vm)
    a.step(0.02, 0.1, 1.0, 4)
    ref = a.get_state()
    a.close()
    b = J.Solver(cfg)
    b.set_state(pp, vp, pm, vm)
    with pytest.raises(J.JanusError):
        b.get_accel()
    b.step(0.02, 0.1, 1.0, 1)
    cur = list(b.get_state())
    acc = list(b.get_accel())
    for _ in range(3):
        b.set_state(*cur)
        b.set_accel(*acc)
        back = b.get_accel()
        assert np.array_equal(back[0], acc[0]) and np.array_equal(back[1], acc[1])
        b.step(0.02, 0.1, 1.0, 1)
        b.get_state(out=cur)
        b.get_accel(out=acc)
    t = b.timings()
    b.close()
    for k in (0, 2):
        d = np.abs(cur[k].astype(np.float64) - ref[k])
        d = np.minimum(d, L - d)
        assert d.max() <= 1e-5 * L
    for k in (1, 3):
        rms = np.sqrt(np.mean(np.sum(ref[k].astype(np.float64) ** 2, axis=1)))
        assert np.abs(cur[k] - ref[k]).max() <= 1e-4 * rms
    # one force pass per step: the stored accelerations were used
    assert t["launches"] < 25


def test_step_grouping_does_not_change_the_trajectory():
    """With Hubble drag on, one call of four steps and four calls of one
    step give the same trajectory to rounding: the fused kick between two
    steps is the closing half kick followed by the opening one."""
    from janus_treepm import ics
    L, n = 60.0, 16
    pp, vp, pm, vm = ics.zeldovich_lattice(n, L, seed=8)
    cfg = J.Config(box_L=L, pm_grid=32, softening=0.05, mu=3.0, theta=0.1)
    out = []
    for calls in (1, 4):
        s = J.Solver(cfg)
        s.set_state(pp, vp, pm, vm)
        for _ in range(calls):
            s.step(0.02, 0.3, 1.0, 4 // calls)
        out.append(s.get_state())
        s.close()
    for k in (1, 3):
        rms = np.sqrt(np.mean(np.sum(out[0][k].astype(np.float64) ** 2, axis=1)))
        assert np.abs(out[0][k] - out[1][k]).max() <= 1e-5 * rms


@pytest.mark.parametrize("mode", [J.JT_ACCURATE, J.JT_RCOMPAT])
def test_step_host_is_the_round_trip_in_one_call(mode):
    """jt_step_host (upload, one step, download in place; in accurate mode
    the positions come back during the force pass) follows the
    device-resident trajectory like the five separate calls, with the same
    bars; the accelerations it hands back are the ones the next step starts
    from.  Arrays of the wrong type are refused."""
    from janus_treepm import ics
    L, n = 60.0, 20
    pp, vp, pm, vm = ics.zeldovich_lattice(n, L, seed=6)
    cfg = J.Config(box_L=L, pm_grid=32, softening=0.05, mu=3.0, theta=0.1, mode=mode)
    a = J.Solver(cfg)
    a.set_state(pp, vp, pm, vm)
    a.step(0.02, 0.1, 1.0, 4)
    ref = a.get_state()
    ref_acc = a.get_accel()
    a.close()
    b = J.Solver(cfg)
    b.set_state(pp, vp, pm, vm)
    b.step(0.02, 0.1, 1.0, 1)
    cur = [np.ascontiguousarray(x) for x in b.get_state()]
    acc = [np.ascontiguousarray(x) for x in b.get_accel()]
    for _ in range(3):
        b.step_host(cur[0], cur[1], acc[0], cur[2], cur[3], acc[1], 0.02, 0.1, 1.0)
    with pytest.raises(ValueError):
        b.step_host(cur[0].astype(np.float64), cur[1], acc[0], cur[2], cur[3], acc[1], 0.02)
    with pytest.raises(J.JanusError):
        b.step_host(cur[0], cur[1], None, cur[2], cur[3], acc[1], 0.02)
    # the handle holds the same state as the host arrays
    st = b.get_state()
    b.close()
    for k in (0, 2):
        d = np.abs(cur[k].astype(np.float64) - ref[k])
        d = np.minimum(d, L - d)
        assert d.max() <= 1e-5 * L
        assert np.array_equal(st[k], cur[k])
    for k in (1, 3):
        rms = np.sqrt(np.mean(np.sum(ref[k].astype(np.float64) ** 2, axis=1)))
        assert np.abs(cur[k] - ref[k]).max() <= 1e-4 * rms
    for s in (0, 1):
        rms = np.sqrt(np.mean(np.sum(ref_acc[s].astype(np.float64) ** 2, axis=1)))
        assert np.abs(acc[s] - ref_acc[s]).max() <= 1e-4 * rms
