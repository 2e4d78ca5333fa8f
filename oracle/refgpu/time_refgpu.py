"""Time the reference's GPU TreePM step (its own kernels, oracle/_ref/
libref_gpu.so, built by `make -C oracle refgpu`) on the 2x224^3 workload.

TEST INFRASTRUCTURE ONLY: a yardstick for the engine's kernels on the same
GPU.  The workload is the engine bench's (seeded Zel'dovich lattice, L = 250
Mpc, PM 512^3, theta 0.5, r_cut = 4.5 x 1.25 cells, softening spacing/30,
dt = 0.005, H at z = 4) in the reference's own conventions: one signed array,
one mass per particle, and its integer r_cut / 16-bit theta and softening
packing.  Prints one JSON line.

usage: python oracle/refgpu/time_refgpu.py [--n-side 224] [--grid 512] [--steps 3]
"""
import argparse
import ctypes as C
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "janus-sim_b200"))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n-side", type=int, default=224)
    ap.add_argument("--grid", type=int, default=512)
    ap.add_argument("--steps", type=int, default=3)
    args = ap.parse_args()
    from janus_treepm import ics, expansion
    L = 250.0 * args.n_side / 224.0
    M = args.grid
    n = args.n_side ** 3
    pp, vp, pm, vm = ics.zeldovich_lattice(args.n_side, L, seed=42)
    pos = np.ascontiguousarray(np.concatenate([pp, pm]), np.float32)
    vel = np.ascontiguousarray(np.concatenate([vp, vm]), np.float32)
    sg = np.concatenate([np.ones(n, np.int8), -np.ones(n, np.int8)])
    r_s = 1.25 * L / M
    r_cut = 4.5 * r_s
    eps = (L / (2 * n) ** (1.0 / 3.0)) / 30.0
    H = expansion.state_at_redshift(4.0)[2]
    lib = C.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_gpu.so"))
    vp_ = C.c_void_p
    lib.rg_init.argtypes = [C.c_int, vp_, vp_, vp_, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double]
    lib.rg_step.argtypes = [C.c_double] * 4 + [C.POINTER(C.c_double)] * 3
    p = lambda a: a.ctypes.data_as(vp_)
    rc = lib.rg_init(2 * n, p(pos), p(vel), p(sg), M, L, 0.5, eps, 1.0e-3)
    if rc:
        raise SystemExit(f"rg_init failed: {rc}")
    ms, pmms, bhms = C.c_double(), C.c_double(), C.c_double()
    rc = lib.rg_step(0.005, r_cut, H, 1.0, C.byref(ms), C.byref(pmms), C.byref(bhms))   # warm-up
    if rc:
        raise SystemExit(f"rg_step failed: {rc}")
    tot = pmt = bht = 0.0
    for _ in range(args.steps):
        rc = lib.rg_step(0.005, r_cut, H, 1.0, C.byref(ms), C.byref(pmms), C.byref(bhms))
        if rc:
            raise SystemExit(f"rg_step failed: {rc}")
        tot += ms.value
        pmt += pmms.value
        bht += bhms.value
    K = args.steps
    print(json.dumps({
        "what": "reference GPU TreePM step (its own kernels recompiled for sm_100a, its launch order)",
        "workload": f"2x{args.n_side}^3, L={L:g} Mpc, PM {M}^3 (FP64), theta 0.5, r_cut {r_cut:.4f} "
                    f"(packed as integer {int(r_cut)})",
        "ms_per_step": tot / K, "pm_ms": pmt / K, "short_range_ms": bht / K,
        "particle_steps_per_s": 2 * n * K / (tot * 1e-3), "steps": K}), flush=True)
    lib.rg_free()


if __name__ == "__main__":
    main()
