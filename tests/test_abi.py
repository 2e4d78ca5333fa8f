"""The C ABI boundary, on a machine without a GPU.

* libjanus_treepm.so loads and exports every function declared in
  include/janus_treepm.h;
* the ctypes structs match the header's layouts;
* argument checks return the documented codes before any device work
  (a bad config is JT_EINVAL; with no CUDA device a valid config fails
  loudly with JT_ECUDA -- there is no CPU fallback).
"""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "janus_treepm.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:int|void|double|const char\*)\s+(jt_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    import janus_treepm as J
    L = J.library()
    names = declared_functions()
    assert len(names) >= 15
    for n in names:
        assert hasattr(L, n), n


def test_python_binding_covers_the_header():
    import janus_treepm as J
    assert set(declared_functions()) <= set(J.EXPORTED)


def test_struct_layouts_match_header():
    import janus_treepm as J
    # jt_config (include/janus_treepm.h): box_L 0, pm_grid 8, theta 16 ... G_mass_plus 56,
    # k_min 64, mode 68, integrator 72, pm_order 76, pm_interlace 80, cut_tail_ppm 84,
    # reserved 88..96
    assert C.sizeof(J.jt_config) == 96
    assert J.jt_config.cut_tail_ppm.offset == 84
    assert J.jt_config.G_mass_plus.offset == 56 and J.jt_config.k_min.offset == 64
    assert J.jt_config.pm_order.offset == J.jt_config.integrator.offset + 4
    # 8 doubles, 5 int64 counters, cellwalk_ms, interp_ms
    assert C.sizeof(J.jt_timings) == 8 * 8 + 8 * 5 + 16
    assert J.jt_timings.cellwalk_ms.offset == 8 * 8 + 8 * 5
    assert J.jt_timings.interp_ms.offset == 8 * 8 + 8 * 5 + 8


def test_strerror_and_version():
    import janus_treepm as J
    L = J.library()
    assert L.jt_strerror(0) == b"ok"
    assert L.jt_strerror(-1) == b"invalid argument"
    assert L.jt_strerror(-4) == b"device wait timed out"
    assert L.jt_strerror(-99) == b"unknown error"
    assert b"sm_100a" in L.jt_version()


@pytest.mark.parametrize("field,value", [("box_L", -1.0), ("pm_grid", 48), ("pm_grid", 2048),
                                         ("theta", -0.1), ("r_cut", 40.0), ("r_s", 0.0),
                                         ("G_mass_plus", 0.0), ("mode", 7), ("integrator", 9),
                                         ("pm_order", 5), ("pm_order", 1), ("pm_interlace", 3),
                                         ("k_min", -1), ("cut_tail_ppm", -1),
                                         ("cut_tail_ppm", 1000000)])
def test_invalid_config_is_rejected_before_device_work(field, value):
    import janus_treepm as J
    cfg = J.Config(box_L=64.0, pm_grid=64).to_c()
    setattr(cfg, field, value)
    h = C.c_void_p()
    assert J.library().jt_create(C.byref(cfg), C.byref(h)) == J.JT_EINVAL
    assert not h.value


def test_null_arguments():
    import janus_treepm as J
    L = J.library()
    assert L.jt_create(None, None) == J.JT_EINVAL
    assert L.jt_accel(None, None, None, 0) == J.JT_EINVAL
    assert L.jt_step(None, 0.1, 0.0, 1.0, 1) == J.JT_EINVAL
    assert L.jt_get_timings(None, None) == J.JT_EINVAL
    assert L.jt_set_screening(None, 2.0, 0.0) == J.JT_EINVAL
    assert L.jt_batch_set_screening(None, 0, 2.0, 0.0) == J.JT_EINVAL
    assert L.jt_batch_prepare(None, 64) == J.JT_EINVAL
    L.jt_destroy(None)  # no-op


def test_no_cpu_fallback_without_a_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    import janus_treepm as J
    with pytest.raises(J.JanusError) as e:
        J.Solver(J.Config(box_L=64.0, pm_grid=64))
    assert e.value.code == J.JT_ECUDA


def test_config_defaults_follow_the_workload_convention():
    import janus_treepm as J
    c = J.Config(box_L=250.0, pm_grid=512).resolved()
    assert abs(c.r_s - 1.25 * 250.0 / 512) < 1e-12
    assert abs(c.r_cut - 4.5 * c.r_s) < 1e-12


def test_batch_estimate_needs_no_device():
    import janus_treepm as J
    cfg = J.Config(box_L=100.0, pm_grid=64)
    p1, s1 = J.Batch.estimate(cfg, 10_000, 10_000)
    p2, s2 = J.Batch.estimate(cfg, 20_000, 20_000)
    assert 0 < p1 < p2 and 0 < s1 < s2
    # persistent state: 5 float4 + 2 int per particle, plus the k tables
    assert p1 == 20_000 * (5 * 16 + 8) + 2 * 64 * 16
    bad = J.Config(box_L=100.0, pm_grid=64, mode=J.JT_RCOMPAT).resolved().to_c()
    a, b = C.c_size_t(), C.c_size_t()
    assert J.library().jt_batch_estimate(C.byref(bad), 10, 10, C.byref(a), C.byref(b)) == J.JT_EINVAL


def test_server_rejects_bad_arguments_without_a_device():
    import janus_treepm as J
    L = J.library()
    h = C.c_void_p()
    assert L.jt_server_create(0, C.byref(h)) == J.JT_EINVAL
    assert L.jt_server_poll(None, None) == J.JT_EINVAL
    assert L.jt_server_request(None, 0, 0.0) == J.JT_EINVAL
    L.jt_server_destroy(None)
