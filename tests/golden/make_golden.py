"""Generate the golden fixtures from the reference's own kernels.

Run from the repository root after `make -C oracle ref` (needs the reference
checkout; oracle/_ref/libref_twopass.so is its CUDA kernel text compiled for
the host CPU):

    python tests/golden/make_golden.py

Every array in the fixtures is produced by the reference kernels
(compute_morton_f32, radix_histogram/prefix_sum/scatter, build_bvh_tp,
init_leaves_tp, reduce_tp, cic_scatter, apply_green_kernel, cic_gather,
forces_treepm_short_range; src/nbody_gpu_twopass.rs and cuda/cufft_wrapper.cu)
running on inputs drawn here from fixed seeds.  The only host-side steps
restated here are the ones the reference performs in Rust: the 16-bit
parameter packing and the inverse FFT between the Green's-function kernel and
the gather (numpy's f64 inverse real FFT stands in for cuFFT Z2D; the
normalisation kernel is the reference's).
"""
import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402


def ref_tree(pos, box_half, mass):
    R = O.ref()
    n = len(pos)
    keys = np.zeros(n, np.uint64)
    idx = np.zeros(n, np.int32)
    R.ref_morton(np.ascontiguousarray(pos, np.float32).ravel(), n, np.float32(box_half), keys, idx)
    skeys = keys.copy()
    vals = np.arange(n, dtype=np.int32)
    R.ref_radix_sort(skeys, vals, n)
    nn = 2 * n - 1
    left = np.zeros(nn, np.int32)
    right = np.zeros(nn, np.int32)
    parent = np.full(nn, -1, np.int32)
    rl = np.zeros(n, np.int32)
    rr = np.zeros(n, np.int32)
    R.ref_karras(skeys, n, left, right, parent, rl, rr)
    npos = np.zeros(7 * nn, np.float32)
    nm = np.zeros(nn, np.float32)
    ty = np.zeros(nn, np.int32)
    ps = np.ascontiguousarray(pos[vals], np.float32)
    R.ref_leaves_reduce(ps.ravel(), n, np.float32(box_half), np.float32(mass), left, right, parent,
                        rl, rr, npos, nm, ty)
    return dict(pos=pos.astype(np.float32), keys=skeys, perm=vals, left=left[:n - 1],
                right=right[:n - 1], parent=parent, rl=rl[:n - 1], rr=rr[:n - 1],
                node_pos=npos.reshape(nn, 7), node_mass=nm, types=ty, box_half=np.float32(box_half),
                mass=np.float32(mass))


def ref_pm(pos, sg, M, L, g_const, r_s, k_min):
    R = O.ref()
    n = len(pos)
    G = M ** 3
    rp = np.zeros(G)
    rm = np.zeros(G)
    bh, inv_cell, cell = np.float32(L / 2), np.float32(M / L), np.float32(L / M)
    R.ref_cic_scatter(pos.ravel(), sg, rp, rm, n, M, bh, inv_cell)
    phis = []
    for rho in (rp, rm):
        half = np.fft.rfftn(rho.reshape(M, M, M))
        h = np.ascontiguousarray(np.stack([half.real, half.imag], -1)).ravel()
        R.ref_apply_green(h, M, M, M, 2 * np.pi / L, g_const, r_s, k_min)
        hc = h.reshape(M, M, M // 2 + 1, 2)
        # unnormalised Z2D (numpy normalises: undo), then the reference's normalize_kernel
        phi = np.fft.irfftn(hc[..., 0] + 1j * hc[..., 1], s=(M, M, M), axes=(0, 1, 2)).ravel() * G
        phi = np.ascontiguousarray(phi)
        R.ref_normalize(phi, G, 1.0 / G)
        phis.append(phi)
    f = np.zeros(3 * n, np.float32)
    R.ref_cic_gather(pos.ravel(), sg, phis[0], phis[1], f, n, M, bh, inv_cell, cell)
    return rp, rm, phis[0], phis[1], f.reshape(n, 3)


def ref_short(pos_all, sg, trees, theta, eps, r_cut, L):
    R = O.ref()
    n = len(pos_all)
    a, b = C.c_float(), C.c_float()
    R.ref_pack_params(theta, eps, r_cut, L, C.byref(a), C.byref(b))
    acc = np.zeros(3 * n, np.float32)
    for sgn, T in zip((1, -1), trees):
        R.ref_short_range(pos_all.ravel(), sg, T["node_pos"].ravel(), T["node_mass"],
                          np.concatenate([T["left"], np.zeros(n, np.int32)]).astype(np.int32)[:len(T["node_mass"])],
                          np.concatenate([T["right"], np.zeros(n, np.int32)]).astype(np.int32)[:len(T["node_mass"])],
                          T["types"], acc, n if sgn > 0 else -n, a.value, b.value)
    return acc.reshape(n, 3)


def ref_screened(pos_all, sg, trees, theta, eps, lambda_0, z, L):
    """forces_twopass_warpcoherent_screening over both trees (+ overwrites, -
    accumulates), packed as compute_short_range_forces packs it."""
    R = O.ref()
    n = len(pos_all)
    a, b = C.c_float(), C.c_float()
    R.ref_pack_screening(theta, eps, lambda_0, z, L, C.byref(a), C.byref(b))
    acc = np.zeros(3 * n, np.float32)
    for sgn, T in zip((1, -1), trees):
        nn = len(T["node_mass"])
        left = np.concatenate([T["left"], np.full(nn, -1, np.int32)])[:nn].astype(np.int32)
        right = np.concatenate([T["right"], np.full(nn, -1, np.int32)])[:nn].astype(np.int32)
        R.ref_screening(pos_all.ravel(), sg, T["node_pos"].ravel(), T["node_mass"], left, right,
                        T["types"], acc, n, sgn, a.value, b.value)
    return acc.reshape(n, 3)


def screened_fixture():
    """PM + Yukawa-screened walk (lambda_0 > 0.01 branch) on a mixed-sign
    array; theta and softening chosen so that rounding and truncation of the
    1e-3 packing differ."""
    rng = np.random.default_rng(20261203)
    n, M, L = 1100, 16, 32.0
    pos = ((rng.random((n, 3)) - 0.5) * L).astype(np.float32)
    sg = np.where(rng.random(n) < 0.4, 1, -1).astype(np.int8)
    theta, eps, r_cut, mf, lambda_0, z = 0.5497, 0.0508, 5.7, 0.02, 1.93, 0.8
    g_const = mf / (L / M) ** 3
    _, _, _, _, fpm = ref_pm(pos, sg, M, L, g_const, r_cut / 3.0, 0)
    trees = [ref_tree(np.ascontiguousarray(pos[sg == s]), L / 2, mf) for s in (1, -1)]
    fsc = ref_screened(pos, sg, trees, theta, eps, lambda_0, z, L)
    np.savez_compressed(os.path.join(HERE, "screened_mixed_1100.npz"), pos=pos, signs=sg, M=M, L=L,
                        theta=theta, eps=eps, r_cut=r_cut, mass_factor=mf, lambda_0=lambda_0, z=z,
                        pm_forces=fpm, screened=fsc, total=(fsc + fpm).astype(np.float32))


def main():
    out = {}
    rng = np.random.default_rng(20260101)
    L = 64.0
    # 1. uniform species array
    pos = ((rng.random((2000, 3)) - 0.5) * L).astype(np.float32)
    np.savez_compressed(os.path.join(HERE, "tree_uniform_2000.npz"), **ref_tree(pos, L / 2, 0.25))
    # 2. Morton-cell collisions (index tie-break)
    cell = L / 1024
    pos = ((rng.random((1500, 3)) - 0.5) * L).astype(np.float32)
    pos = ((np.floor(pos / (128 * cell)) + 0.5) * 128 * cell).astype(np.float32)  # 512 cells
    np.savez_compressed(os.path.join(HERE, "tree_collide_1500.npz"), **ref_tree(pos, L / 2, 0.25))
    # 3. PM + short-range walk on a mixed-sign array (warp groups straddle species)
    n, M, L2 = 1200, 16, 32.0
    pos = ((rng.random((n, 3)) - 0.5) * L2).astype(np.float32)
    sg = np.where(rng.random(n) < 0.45, 1, -1).astype(np.int8)
    theta, eps, r_cut, mf = 0.5, 0.05, 5.7, 0.02
    g_const = mf / (L2 / M) ** 3
    rp, rm, pp, pmn, fpm = ref_pm(pos, sg, M, L2, g_const, r_cut / 3.0, 0)
    trees = [ref_tree(np.ascontiguousarray(pos[sg == s]), L2 / 2, mf) for s in (1, -1)]
    fsr = ref_short(pos, sg, trees, theta, eps, r_cut, L2)
    np.savez_compressed(os.path.join(HERE, "forces_mixed_1200.npz"), pos=pos, signs=sg, M=M, L=L2,
                        theta=theta, eps=eps, r_cut=r_cut, mass_factor=mf, rho_plus=rp,
                        rho_minus=rm, phi_plus=pp, phi_minus=pmn, pm_forces=fpm, short=fsr,
                        total=(fsr + fpm).astype(np.float32))
    # 4. k_min filter on the Green's function
    rp2, rm2, pp2, pm2, fpm2 = ref_pm(pos, sg, M, L2, g_const, r_cut / 3.0, 3)
    np.savez_compressed(os.path.join(HERE, "pm_kmin3_1200.npz"), pos=pos, signs=sg, M=M, L=L2,
                        g_const=g_const, r_s=r_cut / 3.0, phi_plus=pp2, phi_minus=pm2,
                        pm_forces=fpm2)
    # 5. Yukawa-screened walk
    screened_fixture()
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
