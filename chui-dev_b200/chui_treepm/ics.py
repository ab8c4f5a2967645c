"""Seeded synthetic particle sets for the TreePM benchmarks and tests.

The reference reads external monofonIC/GADGET HDF5 initial conditions
(README.md:85-103), none of which ship with it. These generators stand in for
them with the shapes, sizes and distributions the benchmark configurations
name:

* ``zeldovich_lattice`` -- uniform lattice plus a Gaussian-random Zel'dovich
  displacement field drawn from P(k) ~ k^n (n = -2 by default), scaled to a
  requested rms displacement in lattice spacings; velocities proportional to
  the displacement.
* ``nfw_halos`` -- isotropic NFW halos with log-uniform masses, uniform
  concentrations and virial radii ~ M^(1/3) (the same sampling scheme as the
  reference's tools/generate_clustered_dmo_box.py:34-57: radii by inverse CDF of
  ln(1+x) - x/(1+x), isotropic directions).
* ``clustered_box`` -- halos plus a displaced lattice for the remainder.

All positions are FP64 and canonical in [0, L).
"""
from __future__ import annotations

import math

import numpy as np


def _canonical(x: np.ndarray, box: float) -> np.ndarray:
    w = np.mod(x, box)
    w[w >= box] = 0.0
    return w


def gaussian_displacement(n_side: int, box: float, rms_spacing: float, seed: int,
                          spectral_index: float = -2.0) -> np.ndarray:
    """Zel'dovich displacement field psi (3, n_side^3) with rms |psi| equal to
    rms_spacing * (box / n_side)."""
    rng = np.random.default_rng(seed)
    noise = rng.standard_normal((n_side, n_side, n_side))
    dk = np.fft.rfftn(noise)
    k1 = np.fft.fftfreq(n_side) * n_side
    kz = np.fft.rfftfreq(n_side) * n_side
    kx, ky, kzz = np.meshgrid(k1, k1, kz, indexing="ij")
    k2 = kx * kx + ky * ky + kzz * kzz
    k2[0, 0, 0] = 1.0
    amp = np.power(k2, spectral_index / 4.0)  # sqrt(P(k)) = k^(n/2)
    amp[0, 0, 0] = 0.0
    dk *= amp
    psi = []
    for comp in (kx, ky, kzz):
        # psi_k = i k delta_k / k^2 (displacement is the gradient of the potential)
        pk = 1j * comp * dk / k2
        psi.append(np.fft.irfftn(pk, s=(n_side, n_side, n_side), axes=(0, 1, 2)).ravel())
    psi = np.stack(psi)
    rms = math.sqrt(float(np.mean(np.sum(psi * psi, axis=0))))
    spacing = box / n_side
    if rms > 0:
        psi *= rms_spacing * spacing / rms
    return psi


def zeldovich_lattice(n_side: int, box: float, rms_spacing: float, seed: int,
                      velocity_factor: float = 1.0, spectral_index: float = -2.0):
    """Lattice + Zel'dovich displacements. Returns x, y, z, vx, vy, vz (FP64)."""
    spacing = box / n_side
    g = (np.arange(n_side, dtype=np.float64) + 0.5) * spacing
    qx, qy, qz = np.meshgrid(g, g, g, indexing="ij")
    psi = gaussian_displacement(n_side, box, rms_spacing, seed, spectral_index)
    x = _canonical(qx.ravel() + psi[0], box)
    y = _canonical(qy.ravel() + psi[1], box)
    z = _canonical(qz.ravel() + psi[2], box)
    v = velocity_factor * psi
    return x, y, z, v[0].copy(), v[1].copy(), v[2].copy()


def _nfw_radius_table(c: float, samples: int = 2048):
    x = np.linspace(0.0, c, samples)
    m = np.log1p(x) - x / (1.0 + x)
    return x, m / m[-1]


def nfw_halos(n_particles: int, n_halos: int, box: float, mass_decades: float, seed: int,
              conc_range=(4.0, 12.0), overdensity: float = 200.0, total_particles: int | None = None):
    """Sample n_particles equal-mass particles into n_halos NFW halos.

    Halo masses are log-uniform over `mass_decades`; particles are apportioned
    by mass. Virial radius from M = overdensity * rho_mean * 4/3 pi R^3, with
    rho_mean the mean density of the whole box (total_particles in volume box^3).
    """
    rng = np.random.default_rng(seed)
    total = total_particles if total_particles is not None else n_particles
    logm = rng.uniform(0.0, mass_decades, n_halos)
    w = np.power(10.0, logm)
    counts = np.floor(w / w.sum() * n_particles).astype(np.int64)
    rem = n_particles - int(counts.sum())
    if rem > 0:
        order = np.argsort(-w)
        counts[order[:rem]] += 1
    centers = rng.uniform(0.0, box, (n_halos, 3))
    conc = rng.uniform(conc_range[0], conc_range[1], n_halos)
    rho_mean = total / box ** 3
    xs, ys, zs = [], [], []
    for h in range(n_halos):
        nh = int(counts[h])
        if nh == 0:
            continue
        r_vir = (3.0 * nh / (4.0 * math.pi * overdensity * rho_mean)) ** (1.0 / 3.0)
        c = conc[h]
        tx, tm = _nfw_radius_table(c)
        u = rng.uniform(0.0, 1.0, nh)
        r = np.interp(u, tm, tx) * (r_vir / c)
        mu = rng.uniform(-1.0, 1.0, nh)
        phi = rng.uniform(0.0, 2.0 * math.pi, nh)
        s = np.sqrt(1.0 - mu * mu)
        xs.append(centers[h, 0] + r * s * np.cos(phi))
        ys.append(centers[h, 1] + r * s * np.sin(phi))
        zs.append(centers[h, 2] + r * mu)
    x = _canonical(np.concatenate(xs), box)
    y = _canonical(np.concatenate(ys), box)
    z = _canonical(np.concatenate(zs), box)
    return x, y, z


def clustered_box(n_total: int, box: float, halo_fraction: float, n_halos: int, mass_decades: float,
                  lattice_rms_spacing: float, seed: int):
    """Halo particles plus a Zel'dovich-displaced lattice for the remainder.

    The lattice part uses the largest cube n_side^3 <= (1-halo_fraction) n_total;
    the halo part gets the rest, so the total is exactly n_total.
    Returns x, y, z, vx, vy, vz.
    """
    n_lat_side = int(math.floor(((1.0 - halo_fraction) * n_total) ** (1.0 / 3.0) + 1e-9))
    n_lat = n_lat_side ** 3
    n_halo = n_total - n_lat
    lx, ly, lz, lvx, lvy, lvz = zeldovich_lattice(n_lat_side, box, lattice_rms_spacing, seed)
    hx, hy, hz = nfw_halos(n_halo, n_halos, box, mass_decades, seed + 7919, total_particles=n_total)
    x = np.concatenate([lx, hx])
    y = np.concatenate([ly, hy])
    z = np.concatenate([lz, hz])
    zeros = np.zeros(n_halo)
    vx = np.concatenate([lvx, zeros])
    vy = np.concatenate([lvy, zeros])
    vz = np.concatenate([lvz, zeros])
    # shuffle so the input order carries no spatial information
    perm = np.random.default_rng(seed + 104729).permutation(n_total)
    return x[perm], y[perm], z[perm], vx[perm], vy[perm], vz[perm]
