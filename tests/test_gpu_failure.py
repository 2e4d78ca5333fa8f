"""Failure detection on the GPU without a fault.

Every device-side wait in the library is bounded: the onesweep sort's
decoupled look-back gives up after a fixed number of polls of an empty status
word, sets an error bit and lets the kernel finish; the host reads the bit and
returns JT_ETIMEDOUT.  jt_wait_probe runs that same wait on a status word
that nothing publishes.  The test checks that it times out, reports it, and
that the context still computes forces afterwards.
"""
import ctypes as C

import numpy as np
import pytest

import janus_treepm as J

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_reports():
    flag = C.c_int(-1)
    rc = J.library().jt_wait_probe(1 << 16, C.byref(flag))
    assert rc == J.JT_ETIMEDOUT and flag.value == 1
    # the context is intact: a force evaluation still works
    rng = np.random.default_rng(1)
    pp = rng.uniform(-16, 16, (2000, 3)).astype(np.float32)
    pm = rng.uniform(-16, 16, (2000, 3)).astype(np.float32)
    s = J.Solver(J.Config(box_L=32.0, pm_grid=32, softening=0.05))
    s.set_state(pp, None, pm, None)
    ap, am = s.accel()
    assert np.all(np.isfinite(ap)) and np.all(np.isfinite(am))
    s.close()


def test_probe_rejects_bad_limits():
    flag = C.c_int()
    assert J.library().jt_wait_probe(0, C.byref(flag)) == J.JT_EINVAL
    assert J.library().jt_wait_probe(1 << 25, C.byref(flag)) == J.JT_EINVAL
