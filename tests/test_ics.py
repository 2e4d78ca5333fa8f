"""Device Zel'dovich lattice ICs (jt_ics.cu).

CPU: the generator's Philox4x32-10 stream against the published known-answer
vectors (Salmon et al., SC'11, Random123 distribution), both the library's
host copy and the oracle's numpy restatement; the oracle's field properties.
GPU: the device ICs against the FP64 oracle fed the same noise (positions
within 1e-4 lattice spacings plus float32 rounding, velocities within 1e-4 of
the largest), and the handle / batch entry points load exactly those arrays."""
import os
import sys

import numpy as np
import pytest

import janus_treepm as J

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

KAT = [((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
       ((0xFFFFFFFF,) * 4, (0xFFFFFFFF, 0xFFFFFFFF), (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
       ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
        (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1))]


@pytest.mark.parametrize("ctr,key,want", KAT)
def test_philox_known_answers(ctr, key, want):
    assert J.philox4x32_10(ctr, key) == want
    got = O.philox4x32_10(*[np.array([c], np.uint32) for c in ctr], *key)
    assert tuple(int(x[0]) for x in got) == want


def test_oracle_field_properties():
    n, L = 16, 40.0
    a = L / n
    pp, vp, pm, vm = O.zeldovich_philox(n, L, seed=5)
    assert np.all(np.abs(pp) <= L / 2) and np.all(np.abs(pm) <= L / 2)
    dp = vp / 0.05
    assert np.sqrt(np.mean(np.sum(dp ** 2, 1))) == pytest.approx(0.3 * a, rel=1e-12)
    assert np.abs(dp.mean(0)).max() < 1e-12 * a          # no k = 0 mode
    # delta- = -delta+: the m- field is minus the m+ field half a cell away;
    # with the spectrum's smooth cut the two lattices' fields are close
    dm = vm / 0.05
    assert np.corrcoef(dp[:, 0], -dm[:, 0])[0, 1] > 0.8


@pytest.mark.gpu
@pytest.mark.parametrize("n,L,seed", [(32, 50.0, 42), (48, 120.0, 7), (31, 30.0, 3)])
def test_device_ics_match_oracle(n, L, seed):
    pp, vp, pm, vm = J.zeldovich_device(n, L, seed=seed)
    op, ovp, om, ovm = O.zeldovich_philox(n, L, seed=seed)
    a = L / n
    tol = 1e-4 * a + 4 * np.spacing(np.float32(L / 2))
    for got, ref in ((pp, op), (pm, om)):
        d = np.abs(got.astype(np.float64) - ref)
        d = np.minimum(d, L - d)
        assert d.max() <= tol, d.max()
    for got, ref in ((vp, ovp), (vm, ovm)):
        assert np.abs(got - ref).max() <= 1e-4 * np.abs(ref).max()


@pytest.mark.gpu
def test_handle_and_batch_load_the_generated_state():
    n, L = 24, 40.0
    pp, vp, pm, vm = J.zeldovich_device(n, L, seed=11)
    cfg = J.Config(box_L=L, pm_grid=32, softening=0.05, mu=5.0)
    s = J.Solver(cfg)
    s.set_state_zeldovich(n, seed=11)
    gp, gvp, gm, gvm = s.get_state()
    for x, y in ((gp, pp), (gvp, vp), (gm, pm), (gvm, vm)):
        assert np.array_equal(x, y)
    a1 = s.accel()
    s.set_state(pp, vp, pm, vm)
    a2 = s.accel()
    # the deposit accumulates with float atomics: equal to rounding
    for x, y in zip(a1, a2):
        assert np.abs(x - y).max() <= 1e-5 * np.abs(y).max()
    s.close()
    B = J.Batch()
    bid = B.add_zeldovich(cfg, n, seed=11)
    bp, bvp, bm, bvm = B.get_state(bid)
    for x, y in ((bp, pp), (bvp, vp), (bm, pm), (bvm, vm)):
        assert np.array_equal(x, y)
    B.close()
