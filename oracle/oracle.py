"""ctypes bindings for the CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs import
this module.  It loads oracle/liboracle.so (C restatements of the reference
path plus the FP64 Ewald oracles) and, when present, oracle/_ref/
libref_twopass.so (the reference's own CUDA kernel source compiled for the
host CPU).  Both are built by `make -C oracle` / `make -C oracle ref`.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None
_ref = None

f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
i8p = np.ctypeslib.ndpointer(np.int8, flags="C_CONTIGUOUS")
i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
I64, I32, F32, F64 = C.c_int64, C.c_int, C.c_float, C.c_double


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle not built: run `make -C oracle`")
        L = C.CDLL(path)
        sig = {
            "orc_morton30": [f32p, I64, F32, u32p],
            "orc_sort_keys": [u32p, I64, i32p],
            "orc_karras": [u32p, i32p, I64, i32p, i32p, i32p, i32p, i32p],
            "orc_leaves_reduce": [f32p, I64, F32, F32, i32p, i32p, i32p, f32p, f32p, i32p],
            "orc_ref_cic_scatter": [f32p, i8p, I64, I32, F32, F32, f64p, f64p],
            "orc_ref_poisson": [f64p, f64p, I32, F64, F64, F64, I32],
            "orc_ref_cic_gather": [f32p, i8p, I64, I32, F32, F32, F32, f64p, f64p, f32p],
            "orc_ref_pm_forces": [f32p, i8p, I64, I32, F64, F64, F64, I32, f32p],
            "orc_ref_quantize": [F64, F64, F64, F64, C.POINTER(F32), C.POINTER(F32),
                                 C.POINTER(F32), C.POINTER(F32)],
            "orc_ref_short_range": [f32p, i8p, I64, I32, f32p, f32p, i32p, i32p, i32p,
                                    F32, F32, F32, F32, I32, f32p],
            "orc_ref_total_forces": [f32p, i8p, I64, I32, F64, F64, F64, F64, F64, I32, f32p],
            "orc_ref_screen_quantize": [F64, F64, F64, F64, F64, C.POINTER(F32), C.POINTER(F32),
                                        C.POINTER(F32), C.POINTER(F32)],
            "orc_ref_screened_walk": [f32p, i8p, I64, I32, f32p, f32p, i32p, i32p, i32p,
                                      F32, F32, F32, F32, I32, f32p],
            "orc_ref_total_forces_screened": [f32p, i8p, I64, I32, F64, F64, F64, F64, F64, I32,
                                              F64, F64, f32p],
            "orc_cpu_treepm_forces": [f64p, f64p, i8p, I64, F64, I32, F64, F64, F64, f64p],
            "orc_cpu_treepm_last_times": [C.POINTER(F64), C.POINTER(F64)],
            "orc_ewald_forces": [f64p, f64p, i8p, I64, i64p, I64, F64, F64, F64, F64, F64, f64p],
            "orc_ewald_long": [f64p, f64p, i8p, I64, i64p, I64, F64, F64, F64, f64p],
            "orc_ewald_short": [f64p, f64p, i8p, I64, i64p, I64, F64, F64, F64, F64, f64p],
            "orc_acc_pm_forces": [f64p, f64p, i8p, I64, I32, F64, F64, I32, f64p],
            "orc_acc_pm_grids": [f64p, f64p, i8p, I64, I32, F64, F64, I32, f64p, f64p, f64p],
            "orc_acc_pm_forces2": [f64p, f64p, i8p, I64, I32, F64, F64, I32, I32, I32, f64p],
            "orc_fft3d": [f64p, I32, I32],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = None
        L.orc_expand10.argtypes = [C.c_uint32]
        L.orc_expand10.restype = C.c_uint32
        _lib = L
    return _lib


_gpu = None


def gpu_lib():
    """The FP64 periodic force oracle on the GPU (oracle/libewald_gpu.so,
    `make -C oracle gpu`): production-size accuracy checks."""
    global _gpu
    if _gpu is None:
        path = os.path.join(HERE, "libewald_gpu.so")
        if not os.path.exists(path):
            raise RuntimeError("GPU oracle not built: run `make -C oracle gpu`")
        G = C.CDLL(path)
        u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")
        G.oge_periodic_forces.argtypes = [f32p, u8p, I64, F64, F64, i64p, I64, F64, F64, F64, F64,
                                          F64, F64, f64p, f64p]
        G.oge_periodic_forces.restype = C.c_int
        _gpu = G
    return _gpu


def periodic_forces_gpu(pos_p, pos_m, m_plus, m_minus, idx, box, eps, r_e, r_s, r_cut,
                        kcut_tol=1e-12):
    """FP64 accelerations of targets idx (rows of [pos_p ; pos_m]) on the GPU.

    Returns (full, split): `full` the periodic sum with Plummer softening
    (Ewald, wide split r_e, real space within 11 r_e < L/2), `split` the
    truncated split model at r_s / r_cut (= ewald_forces(r_s, eps,
    r_trunc=r_cut)).  Positions are the engine's FP32 inputs, taken exactly."""
    pos = np.ascontiguousarray(np.concatenate([np.asarray(pos_p, np.float32).reshape(-1, 3),
                                               np.asarray(pos_m, np.float32).reshape(-1, 3)]))
    n_p = len(np.asarray(pos_p).reshape(-1, 3))
    sp = np.zeros(len(pos), np.uint8)
    sp[n_p:] = 1
    idx = _c(idx, np.int64)
    full = np.zeros((len(idx), 3), np.float64)
    split = np.zeros((len(idx), 3), np.float64)
    r = gpu_lib().oge_periodic_forces(pos.ravel(), sp, len(pos), float(m_plus), -float(m_minus), idx,
                                      len(idx), box, eps, r_e, r_s, r_cut, kcut_tol, full.ravel(),
                                      split.ravel())
    if r != 0:
        raise RuntimeError(f"oge_periodic_forces failed: {r}")
    return full, split


def ref_available():
    return os.path.exists(os.path.join(HERE, "_ref", "libref_twopass.so"))


def ref():
    """The reference kernels compiled for the host (oracle/_ref)."""
    global _ref
    if _ref is None:
        path = os.path.join(HERE, "_ref", "libref_twopass.so")
        if not os.path.exists(path):
            raise RuntimeError("reference harness not built: run `make -C oracle ref`")
        R = C.CDLL(path)
        sig = {
            "ref_morton": [f32p, I32, F32, u64p, i32p],
            "ref_radix_sort": [u64p, i32p, I32],
            "ref_karras": [u64p, I32, i32p, i32p, i32p, i32p, i32p],
            "ref_leaves_reduce": [f32p, I32, F32, F32, i32p, i32p, i32p, i32p, i32p,
                                  f32p, f32p, i32p],
            "ref_cic_scatter": [f32p, i8p, f64p, f64p, I32, I32, F32, F32],
            "ref_cic_gather": [f32p, i8p, f64p, f64p, f32p, I32, I32, F32, F32, F32],
            "ref_apply_green": [f64p, I32, I32, I32, F64, F64, F64, I32],
            "ref_normalize": [f64p, I32, F64],
            "ref_pack_params": [F64, F64, F64, F64, C.POINTER(F32), C.POINTER(F32)],
            "ref_short_range": [f32p, i8p, f32p, f32p, i32p, i32p, i32p, f32p, I32, F32, F32],
            "ref_pack_screening": [F64, F64, F64, F64, F64, C.POINTER(F32), C.POINTER(F32)],
            "ref_screening": [f32p, i8p, f32p, f32p, i32p, i32p, i32p, f32p, I32, I32, F32, F32],
            "ref_drift": [f32p, f32p, F32, F32, I32],
            "ref_kick": [f32p, f32p, F32, I32, F32, F32],
        }
        for name, args in sig.items():
            fn = getattr(R, name)
            fn.argtypes = args
            fn.restype = None
        _ref = R
    return _ref


# ---------------------------------------------------------------- helpers
def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def morton30(pos, box_half):
    pos = _c(pos, np.float32).reshape(-1, 3)
    out = np.empty(len(pos), np.uint32)
    lib().orc_morton30(pos.ravel(), len(pos), np.float32(box_half), out)
    return out


def build_tree(pos, box_half, mass):
    """Reference LBVH over one species (positions in the species' own order).

    Returns a dict with m30 (sorted), perm, pos_sorted, left, right, parent,
    rl, rr, node_pos (2n-1, 7), node_mass, types."""
    pos = _c(pos, np.float32).reshape(-1, 3)
    n = len(pos)
    nn = max(2 * n - 1, 1)
    L = lib()
    m30 = morton30(pos, box_half)
    perm = np.empty(n, np.int32)
    L.orc_sort_keys(m30, n, perm)
    m30s = np.ascontiguousarray(m30[perm])
    pos_s = np.ascontiguousarray(pos[perm])
    left = np.zeros(nn, np.int32)
    right = np.zeros(nn, np.int32)
    parent = np.zeros(nn, np.int32)
    rl = np.zeros(max(n - 1, 1), np.int32)
    rr = np.zeros(max(n - 1, 1), np.int32)
    L.orc_karras(m30s, perm, n, left, right, parent, rl, rr)
    node_pos = np.zeros(7 * nn, np.float32)
    node_mass = np.zeros(nn, np.float32)
    types = np.zeros(nn, np.int32)
    L.orc_leaves_reduce(pos_s.ravel(), n, np.float32(box_half), np.float32(mass),
                        left, right, parent, node_pos, node_mass, types)
    return dict(m30=m30s, perm=perm, pos_sorted=pos_s, left=left, right=right,
                parent=parent, rl=rl[:max(n - 1, 0)], rr=rr[:max(n - 1, 0)],
                node_pos=node_pos.reshape(nn, 7), node_mass=node_mass, types=types)


def ref_quantize(theta, softening, r_cut, box):
    a, b, c, d = F32(), F32(), F32(), F32()
    lib().orc_ref_quantize(theta, softening, r_cut, box, C.byref(a), C.byref(b),
                           C.byref(c), C.byref(d))
    return a.value, b.value, c.value, d.value


def ref_total_forces(pos_all, signs_all, M, box, theta, softening, r_cut,
                     mass_factor, k_min=0):
    """Reference GPU TreePM acceleration (PM + both trees), FP32 out."""
    pos_all = _c(pos_all, np.float32).reshape(-1, 3)
    signs_all = _c(signs_all, np.int8)
    acc = np.zeros((len(pos_all), 3), np.float32)
    lib().orc_ref_total_forces(pos_all.ravel(), signs_all, len(pos_all), M, box,
                               theta, softening, r_cut, mass_factor, k_min, acc.ravel())
    return acc


def ref_screen_quantize(theta, softening, lambda_0, z, box):
    """(theta, softening, 1/lambda, box_half) as the screened walk sees them."""
    a, b, c, d = F32(), F32(), F32(), F32()
    lib().orc_ref_screen_quantize(theta, softening, lambda_0, z, box, C.byref(a), C.byref(b),
                                  C.byref(c), C.byref(d))
    return a.value, b.value, c.value, d.value


def ref_total_forces_screened(pos_all, signs_all, M, box, theta, softening, r_cut,
                              mass_factor, lambda_0, z, k_min=0):
    """Reference GPU TreePM acceleration with Yukawa screening of opposite-sign
    pairs (lambda_0 > 0.01: PM + the full-range screened walk), FP32 out."""
    pos_all = _c(pos_all, np.float32).reshape(-1, 3)
    signs_all = _c(signs_all, np.int8)
    acc = np.zeros((len(pos_all), 3), np.float32)
    lib().orc_ref_total_forces_screened(pos_all.ravel(), signs_all, len(pos_all), M, box, theta,
                                        softening, r_cut, mass_factor, k_min, lambda_0, z,
                                        acc.ravel())
    return acc


def ref_pm_forces(pos_all, signs_all, M, box, mass_factor, r_cut, k_min=0):
    pos_all = _c(pos_all, np.float32).reshape(-1, 3)
    signs_all = _c(signs_all, np.int8)
    out = np.zeros((len(pos_all), 3), np.float32)
    lib().orc_ref_pm_forces(pos_all.ravel(), signs_all, len(pos_all), M, box,
                            mass_factor, r_cut, k_min, out.ravel())
    return out


def cpu_treepm_forces(pos, mass, signs, r_cut, grid, box, theta, softening):
    """Reference CPU TreePM (src/treepm) on all particles; returns (acc, t_update, t_forces)."""
    pos = _c(pos, np.float64).reshape(-1, 3)
    mass = _c(mass, np.float64)
    signs = _c(signs, np.int8)
    acc = np.zeros((len(pos), 3), np.float64)
    L = lib()
    L.orc_cpu_treepm_forces(pos.ravel(), mass, signs, len(pos), r_cut, grid, box,
                            theta, softening, acc.ravel())
    tu, tf = F64(), F64()
    L.orc_cpu_treepm_last_times(C.byref(tu), C.byref(tf))
    return acc, tu.value, tf.value


def ewald_forces(pos, mass, signs, box, r_s, eps, r_trunc=None, idx=None,
                 kcut_tol=1e-12, part="all"):
    """FP64 periodic oracle on targets idx (default all).  part: all|long|short."""
    pos = _c(pos, np.float64).reshape(-1, 3)
    mass = _c(mass, np.float64)
    signs = _c(signs, np.int8)
    n = len(pos)
    idx = np.arange(n, dtype=np.int64) if idx is None else _c(idx, np.int64)
    if r_trunc is None:
        r_trunc = 12.0 * r_s   # S(r) < 1e-14 beyond
    acc = np.zeros((len(idx), 3), np.float64)
    L = lib()
    if part == "all":
        L.orc_ewald_forces(pos.ravel(), mass, signs, n, idx, len(idx), box, r_s, eps,
                           r_trunc, kcut_tol, acc.ravel())
    elif part == "long":
        L.orc_ewald_long(pos.ravel(), mass, signs, n, idx, len(idx), box, r_s, kcut_tol,
                         acc.ravel())
    else:
        L.orc_ewald_short(pos.ravel(), mass, signs, n, idx, len(idx), box, r_s, eps,
                          r_trunc, acc.ravel())
    return acc


def acc_pm_forces(pos, mass, signs, M, box, r_s, k_min=0, order=2, interlace=False):
    """FP64 PM acceleration (long range only) in the accurate formulation."""
    pos = _c(pos, np.float64).reshape(-1, 3)
    mass = _c(mass, np.float64)
    signs = _c(signs, np.int8)
    acc = np.zeros((len(pos), 3), np.float64)
    lib().orc_acc_pm_forces2(pos.ravel(), mass, signs, len(pos), M, box, r_s, k_min, order,
                             2 if interlace else 1, acc.ravel())
    return acc


# ---------------------------------------------------------------------------
# Diagnostics (numpy restatements of the reference's host-side metrics)
# ---------------------------------------------------------------------------
def segregation(pos, signs, box):
    """|COM+ - COM-| / L with plain means (src/nbody_gpu_twopass.rs:5364-5393)."""
    pos = np.asarray(pos, np.float32).astype(np.float64).reshape(-1, 3)
    signs = np.asarray(signs)
    cp = pos[signs > 0].mean(axis=0) if np.any(signs > 0) else np.zeros(3)
    cm = pos[signs < 0].mean(axis=0) if np.any(signs < 0) else np.zeros(3)
    return float(np.linalg.norm(cp - cm) / box)


def segregation_metrics(pos, signs, box, n_cells):
    """compute_segregation_metrics (src/bin/janus_mu19_production.rs:219-276):
    NGP counts of each species on an n_cells^3 grid (cell of a coordinate:
    rem_euclid(x + L/2, L) / cell, truncated, mod n_cells), then
    (Var(n+ - n-) / (mean+ + mean-), Corr(delta+, delta-),
     (Var(n-) - mean-) / mean-)."""
    pos = np.asarray(pos, np.float32).astype(np.float64).reshape(-1, 3)
    signs = np.asarray(signs)
    cell = box / n_cells
    r = np.mod(pos + box / 2.0, box)
    ic = (np.floor(r / cell).astype(np.int64)) % n_cells
    flat = (ic[:, 0] * n_cells + ic[:, 1]) * n_cells + ic[:, 2]
    tot = n_cells ** 3
    n_plus = np.bincount(flat[signs > 0], minlength=tot).astype(np.float64)
    n_minus = np.bincount(flat[signs < 0], minlength=tot).astype(np.float64)
    mp, mm = n_plus.sum() / tot, n_minus.sum() / tot
    diff = n_plus - n_minus - (mp - mm)
    var_diff = np.mean(diff ** 2)
    pois = mp + mm
    dop = var_diff / pois if pois > 0 else 0.0
    dp = (n_plus - mp) / mp if mp > 0 else np.zeros(tot)
    dm = (n_minus - mm) / mm if mm > 0 else np.zeros(tot)
    var_p = np.mean(dp * dp) - np.mean(dp) ** 2
    var_m = np.mean(dm * dm) - np.mean(dm) ** 2
    cov = np.mean(dp * dm) - np.mean(dp) * np.mean(dm)
    corr = cov / (np.sqrt(var_p) * np.sqrt(var_m)) if var_p > 0 and var_m > 0 else 0.0
    var_mc = np.mean((n_minus - mm) ** 2)
    exc = (var_mc - mm) / mm if mm > 0 else 0.0
    return float(dop), float(corr), float(exc)


# ---------------------------------------------------------------- Zel'dovich ICs
def philox4x32_10(c0, c1, c2, c3, k0, k1):
    """Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11), vectorised over
    uint32 counter arrays; keys are Python ints."""
    M0, M1 = np.uint64(0xD2511F53), np.uint64(0xCD9E8D57)
    c = [np.asarray(x, np.uint32) for x in (c0, c1, c2, c3)]
    for _ in range(10):
        p0 = M0 * c[0].astype(np.uint64)
        p1 = M1 * c[2].astype(np.uint64)
        hi0, lo0 = (p0 >> np.uint64(32)).astype(np.uint32), (p0 & np.uint64(0xFFFFFFFF)).astype(np.uint32)
        hi1, lo1 = (p1 >> np.uint64(32)).astype(np.uint32), (p1 & np.uint64(0xFFFFFFFF)).astype(np.uint32)
        c = [hi1 ^ c[1] ^ np.uint32(k0), lo1, hi0 ^ c[3] ^ np.uint32(k1), lo0]
        k0 = (k0 + 0x9E3779B9) & 0xFFFFFFFF
        k1 = (k1 + 0xBB67AE85) & 0xFFFFFFFF
    return c


def zeldovich_philox(n, L, seed=42, rms_frac=0.3, vel_factor=0.05):
    """FP64 restatement of the device Zel'dovich lattice generator: the same
    Philox noise per cell (counter = cell index, key = seed; Box-Muller), the
    spectrum P(k) = A k^-2.5 exp(-(k/k_c)^2) with k_c = pi / (2 a), psi = i k
    / k^2 delta(k) with k = 0 and the Nyquist planes zeroed, psi- = -psi on
    the lattice offset by a/2, rms |psi+| = rms_frac a, v = vel_factor psi.
    Returns (pos_p, vel_p, pos_m, vel_m) as float64 (n^3, 3) arrays, rows in
    lattice order iz n^2 + iy n + ix."""
    n3 = n ** 3
    idx = np.arange(n3, dtype=np.uint64)
    r = philox4x32_10((idx & np.uint64(0xFFFFFFFF)).astype(np.uint32),
                      (idx >> np.uint64(32)).astype(np.uint32), np.zeros(n3, np.uint32),
                      np.zeros(n3, np.uint32), seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF)
    u0 = (r[0].astype(np.float64) + 0.5) * 2.0 ** -32
    u1 = (r[1].astype(np.float64) + 0.5) * 2.0 ** -32
    noise = (np.sqrt(-2.0 * np.log(u0)) * np.cos(2.0 * np.pi * u1)).astype(np.float32)
    dk = np.fft.rfftn(noise.reshape(n, n, n).astype(np.float64))
    a = L / n
    kf = 2.0 * np.pi / L
    k1 = kf * np.where(np.arange(n) <= (n - 1) // 2, np.arange(n), np.arange(n) - n)
    kr = kf * np.arange(n // 2 + 1)
    kz, ky, kx = k1[:, None, None], k1[None, :, None], kr[None, None, :]
    k2 = kz * kz + ky * ky + kx * kx
    kc = 0.5 * np.pi / a
    with np.errstate(divide="ignore", invalid="ignore"):
        amp = np.where(k2 > 0, k2 ** -0.625 * np.exp(-0.5 * k2 / kc ** 2), 0.0)
        inv = np.where(k2 > 0, 1.0 / k2, 0.0)
    if n % 2 == 0:
        nyq = np.zeros((n, n, n // 2 + 1), bool)
        nyq[n // 2, :, :] = True
        nyq[:, n // 2, :] = True
        nyq[:, :, n // 2] = True
        amp = np.where(nyq, 0.0, amp)
    shift = np.exp(1j * 0.5 * a * (kx + ky + kz))
    psi = {}
    for name, kc_ in (("x", kx), ("y", ky), ("z", kz)):
        pk = 1j * kc_ * inv * amp * dk
        psi["p" + name] = np.fft.irfftn(pk, s=(n, n, n), axes=(0, 1, 2)).ravel()
        psi["m" + name] = -np.fft.irfftn(pk * shift, s=(n, n, n), axes=(0, 1, 2)).ravel()
    rms = np.sqrt(np.mean(psi["px"] ** 2 + psi["py"] ** 2 + psi["pz"] ** 2))
    scale = rms_frac * a / rms if rms > 0 else 0.0
    i = np.arange(n3)
    lat = np.stack([i % n, (i // n) % n, i // (n * n)], -1).astype(np.float64)
    out = []
    for sp, off in (("p", 0.0), ("m", 0.5 * a)):
        d = np.stack([psi[sp + "x"], psi[sp + "y"], psi[sp + "z"]], -1) * scale
        pos = (lat + 0.5) * a - 0.5 * L + off + d
        pos = (pos + 0.5 * L) % L - 0.5 * L
        out += [pos, vel_factor * d]
    return tuple(out)


# ---------------------------------------------------------------- energies
def kinetic_energy_unit(vel_p, vel_m):
    """kinetic_energy (src/nbody_gpu_twopass.rs:5070-5077): sum |v|^2 / 2 over
    every particle, unit masses, f64."""
    v = np.concatenate([np.asarray(vel_p, np.float64), np.asarray(vel_m, np.float64)])
    return float(0.5 * np.sum(v * v))


def pe_binding_sampled(pos_p, pos_m, n_sample, softening):
    """potential_energy_binding_sampled (src/nbody_gpu_twopass.rs:5081-5181):
    per species rows i * (n / n_sample) (all rows when n <= n_sample), the
    pair sum -sum_{i<j} 1/sqrt(r^2 + eps^2) with plain differences in f64,
    times n (n - 1) / (ns (ns - 1)).  Returns (pe_plus, pe_minus)."""
    out = []
    for pos in (pos_p, pos_m):
        pos = np.asarray(pos, np.float64)
        n = len(pos)
        if n == 0:
            out.append(0.0)
            continue
        sample = pos if n <= n_sample else pos[np.arange(n_sample) * (n // n_sample)]
        ns = len(sample)
        pe = 0.0
        for i in range(ns - 1):
            d = sample[i + 1:] - sample[i]
            pe -= np.sum(1.0 / np.sqrt(np.sum(d * d, axis=1) + softening * softening))
        scale = (n * (n - 1.0)) / (ns * (ns - 1.0)) if ns > 1 else 1.0
        out.append(pe * scale)
    return tuple(out)


def split_energy(pos, mass, signs, box, r_s, eps, r_cut, kcut_tol=1e-12):
    """FP64 potential energy of the truncated split model (short part shifted
    to zero at r_cut): (U, (U_short, U_long, U_self))."""
    pos = _c(pos, np.float64).reshape(-1, 3)
    mass = _c(mass, np.float64)
    signs = _c(signs, np.int8)
    parts = np.zeros(3)
    L = lib()
    L.orc_split_energy.argtypes = [f64p, f64p, i8p, I64, F64, F64, F64, F64, F64, f64p]
    L.orc_split_energy.restype = F64
    u = L.orc_split_energy(pos.ravel(), mass, signs, len(pos), box, r_s, eps, r_cut, kcut_tol, parts)
    return u, tuple(parts)


def ewald_forces_screened(pos, mass, signs, box, r_s, eps, kappa, r_trunc=None, idx=None,
                          kcut_tol=1e-12):
    """FP64 split model with Yukawa screening (kappa = 1 / lambda) of
    opposite-species pairs; kappa = 0 is ewald_forces."""
    pos = _c(pos, np.float64).reshape(-1, 3)
    mass = _c(mass, np.float64)
    signs = _c(signs, np.int8)
    n = len(pos)
    idx = np.arange(n, dtype=np.int64) if idx is None else _c(idx, np.int64)
    if r_trunc is None:
        r_trunc = 12.0 * r_s
    acc = np.zeros((len(idx), 3), np.float64)
    L = lib()
    L.orc_ewald_forces_screened.argtypes = [f64p, f64p, i8p, I64, i64p, I64, F64, F64, F64, F64, F64,
                                            F64, f64p]
    L.orc_ewald_forces_screened.restype = None
    L.orc_ewald_forces_screened(pos.ravel(), mass, signs, n, idx, len(idx), box, r_s, eps, r_trunc,
                                kappa, kcut_tol, acc.ravel())
    return acc
