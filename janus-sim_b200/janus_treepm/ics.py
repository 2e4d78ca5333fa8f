"""Seeded synthetic initial conditions for the TreePM workloads.

The reference draws its ICs with Rust's StdRng (src/bin/janus_mu19_production.rs
:73-105); that stream cannot be reproduced without its toolchain, and parity
runs feed identical arrays to both sides anyway.  These generators use numpy's
PCG64 (default_rng) so every workload is reproducible from its seed.

* uniform_box       -- N per species uniform in [-L/2, L/2)^3 (small case)
* zeldovich_lattice -- per-species n^3 lattice, the m- lattice offset by half a
  cell, Zel'dovich displacements psi = i k / k^2 delta(k) of a Gaussian field
  with P(k) = A k^-2.5 exp(-(k/k_c)^2), k_c = half the lattice Nyquist
  wavenumber, A set so that rms |psi| = rms_frac * spacing; psi- = -psi
  evaluated at the offset lattice (so delta- = -delta+)
* plummer_spheres   -- clustered data: Plummer spheres (scale radii
  log-uniform), species alternating by sphere, plus a uniform background
"""
import numpy as np


def wrap(x, L):
    """Map positions into [-L/2, L/2)."""
    y = (x + 0.5 * L) % L - 0.5 * L
    return np.where(y >= 0.5 * L, y - L, y)


def uniform_box(n_per_species, L, seed=42):
    rng = np.random.default_rng(seed)
    pp = ((rng.random((n_per_species, 3)) - 0.5) * L).astype(np.float32)
    pm = ((rng.random((n_per_species, 3)) - 0.5) * L).astype(np.float32)
    return pp, pm


def zeldovich_lattice(n_side, L, seed=42, rms_frac=0.3, vel_factor=0.05):
    """Returns (pos_p, vel_p, pos_m, vel_m) float32 arrays of n_side^3 rows.

    Velocities are the Zel'dovich growing mode v = vel_factor * psi (Mpc/Gyr
    per Mpc of displacement)."""
    rng = np.random.default_rng(seed)
    n = n_side
    a = L / n
    noise = rng.standard_normal((n, n, n)).astype(np.float32)
    dk = np.fft.rfftn(noise)
    del noise
    k1 = 2 * np.pi * np.fft.fftfreq(n, d=a)
    kr = 2 * np.pi * np.fft.rfftfreq(n, d=a)
    kz = k1[:, None, None].astype(np.float32)
    ky = k1[None, :, None].astype(np.float32)
    kx = kr[None, None, :].astype(np.float32)
    k2 = kz * kz + ky * ky + kx * kx
    k_nyq = np.pi / a
    k_c = 0.5 * k_nyq
    with np.errstate(divide="ignore", invalid="ignore"):
        kk = np.sqrt(k2)
        amp = np.where(k2 > 0, kk ** (-1.25) * np.exp(-0.5 * (kk / k_c) ** 2), 0.0).astype(np.float32)
        dk *= amp
        inv_k2 = np.where(k2 > 0, 1.0 / k2, 0.0).astype(np.float32)
    # half-cell shift for the m- lattice: exp(i k . (a/2, a/2, a/2))
    shift = np.exp(1j * 0.5 * a * (kx + ky + kz)).astype(np.complex64)
    out = {}
    for name, comp_k in (("x", kx), ("y", ky), ("z", kz)):
        psik = (1j * comp_k * inv_k2 * dk).astype(np.complex64)
        out[name + "p"] = np.fft.irfftn(psik, s=(n, n, n), axes=(0, 1, 2)).astype(np.float32)
        out[name + "m"] = -np.fft.irfftn(psik * shift, s=(n, n, n), axes=(0, 1, 2)).astype(np.float32)
        del psik
    rms = np.sqrt(np.mean(out["xp"] ** 2 + out["yp"] ** 2 + out["zp"] ** 2))
    scale = rms_frac * a / rms
    # lattice coordinates: index (z, y, x) -> position -L/2 + (i + 0.5) a
    g = (np.arange(n, dtype=np.float32) + 0.5) * a - 0.5 * L
    Z, Y, X = np.meshgrid(g, g, g, indexing="ij")
    res = []
    for sp, off in (("p", 0.0), ("m", 0.5 * a)):
        psi = np.stack([out["x" + sp], out["y" + sp], out["z" + sp]], -1).reshape(-1, 3) * scale
        base = np.stack([X, Y, Z], -1).reshape(-1, 3) + off
        pos = wrap(base + psi, L).astype(np.float32)
        vel = (vel_factor * psi).astype(np.float32)
        res += [pos, vel]
    return tuple(res)


def plummer_spheres(n_per_species, L, n_spheres=512, bg_frac=0.2, a_min=0.05, a_max=1.0,
                    seed=42):
    """Clustered data: each species fills its own alternating half of the
    spheres (80%) plus a uniform background (20%)."""
    rng = np.random.default_rng(seed)
    centres = (rng.random((n_spheres, 3)) - 0.5) * L
    scales = np.exp(rng.uniform(np.log(a_min), np.log(a_max), n_spheres))
    out = []
    for sp in (0, 1):
        mine = np.arange(sp, n_spheres, 2)
        n_bg = int(round(bg_frac * n_per_species))
        n_cl = n_per_species - n_bg
        which = mine[rng.integers(0, len(mine), n_cl)]
        u = rng.uniform(1e-6, 1.0, n_cl)
        r = scales[which] / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        r = np.minimum(r, 10.0 * scales[which])
        d = rng.standard_normal((n_cl, 3))
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        cl = centres[which] + d * r[:, None]
        bg = (rng.random((n_bg, 3)) - 0.5) * L
        pos = wrap(np.concatenate([cl, bg]), L).astype(np.float32)
        out.append(pos[rng.permutation(n_per_species)])
    return out[0], out[1]
