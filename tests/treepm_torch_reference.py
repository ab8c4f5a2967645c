"""Independent FP64 torch formulation of the periodic TreePM force and static
KDK, used as the reference gradient for the adjoint kernels (torch autograd
differentiates it; nothing here calls the library's kernels).

It restates the same algorithm as the reference's PM solver and residual tree
force with the tree replaced by the direct sum over all pairs inside r_cut,
which is what the strict walk computes when no node is accepted as a
multipole (internal nodes must satisfy 2h/r < 0.08 to be accepted):
- CIC/TSC deposit and interpolation: pm_solver.cpp:925-951 (stencils),
  :3842-4057 (deposit), :5735-5953 (interpolation);
- Poisson with window deconvolution and Gaussian split filter, spectral
  gradient with the differentiated even-axis Nyquist zeroed:
  pm_solver.cpp:2398-2466, :2557-2706, :4581-4940;
- residual pair kernel (r^2+eps^2)^-3/2 - [erf(q) - 2q e^{-q^2}/sqrt(pi)]/r^3,
  q = r/(2 r_s), with the q < 1/8 series: tree_pm_split_kernel.hpp:66-228;
- static KDK factors: time_integration.cpp:429-441.
"""
from __future__ import annotations

import math

import torch

SQRT_PI_INV = 1.0 / math.sqrt(math.pi)


def _stencil(gp: torch.Tensor, scheme: int):
    """Base cell and weights per axis (differentiable in gp)."""
    if scheme == 0:
        base = torch.floor(gp.detach())
        t = gp - base
        return base.long(), [1.0 - t, t]
    center = torch.floor(gp.detach() + 0.5)
    d = gp - center
    return center.long() - 1, [0.5 * (0.5 - d) ** 2, 0.75 - d * d, 0.5 * (0.5 + d) ** 2]


def _wrap(v: torch.Tensor, L: float) -> torch.Tensor:
    w = torch.fmod(v, L)
    return torch.where(w < 0, w + L, w)


def _cells_weights(pos, mesh, box, scheme):
    out = []
    for a in range(3):
        gp = _wrap(pos[a], box[a]) * (mesh[a] / box[a])
        base, w = _stencil(gp, scheme)
        out.append((base, w))
    return out


def deposit(pos, mass, mesh, box, scheme):
    """Density (mass / cell volume) on the mesh, shape mesh."""
    nx, ny, nz = mesh
    cw = _cells_weights(pos, mesh, box, scheme)
    taps = len(cw[0][1])
    rho = torch.zeros(nx * ny * nz, dtype=torch.float64, device=pos[0].device)
    for a in range(taps):
        ix = (cw[0][0] + a) % nx
        for b in range(taps):
            iy = (cw[1][0] + b) % ny
            for c in range(taps):
                iz = (cw[2][0] + c) % nz
                w = cw[0][1][a] * cw[1][1][b] * cw[2][1][c]
                rho = rho.index_add(0, (ix * ny + iy) * nz + iz, mass * w)
    vol = box[0] * box[1] * box[2] / (nx * ny * nz)
    return (rho / vol).reshape(nx, ny, nz)


def interpolate(grids, pos, mesh, box, scheme):
    nx, ny, nz = mesh
    cw = _cells_weights(pos, mesh, box, scheme)
    taps = len(cw[0][1])
    flat = [g.reshape(-1) for g in grids]
    acc = [0.0, 0.0, 0.0]
    for a in range(taps):
        ix = (cw[0][0] + a) % nx
        for b in range(taps):
            iy = (cw[1][0] + b) % ny
            for c in range(taps):
                iz = (cw[2][0] + c) % nz
                w = cw[0][1][a] * cw[1][1][b] * cw[2][1][c]
                idx = (ix * ny + iy) * nz + iz
                for d in range(3):
                    acc[d] = acc[d] + w * flat[d][idx]
    return acc


def _axis(n, L, half, deconv, expo, device):
    count = n // 2 + 1 if half else n
    i = torch.arange(count, device=device, dtype=torch.float64)
    mode = i if half else torch.where(i <= n // 2, i, i - n)
    k = 2.0 * math.pi / L * mode
    if deconv:
        v = 0.5 * k * L / n
        s = torch.where(v.abs() < 1e-12, torch.ones_like(v), torch.sin(v) / torch.where(v == 0, torch.ones_like(v), v))
        w = s ** expo
    else:
        w = torch.ones_like(k)
    g = k.clone()
    if n % 2 == 0:
        g[n // 2] = 0.0
    return k, w, g


def pm_accel(pos, mass, mesh, box, rs, G, scheme, deconv):
    nx, ny, nz = mesh
    dev = pos[0].device
    expo = 2 if scheme == 0 else 3
    rho = deposit(pos, mass, mesh, box, scheme)
    total = mass.sum()
    rho = rho - total / (box[0] * box[1] * box[2])
    rk = torch.fft.rfftn(rho)
    kx, wx, gx = _axis(nx, box[0], False, deconv, expo, dev)
    ky, wy, gy = _axis(ny, box[1], False, deconv, expo, dev)
    kz, wz, gz = _axis(nz, box[2], True, deconv, expo, dev)
    k2 = kx[:, None, None] ** 2 + ky[None, :, None] ** 2 + kz[None, None, :] ** 2
    tw = wx[:, None, None] * wy[None, :, None] * wz[None, None, :]
    window = 1.0 / torch.clamp(tw * tw, min=1e-12)
    pref = -4.0 * math.pi * G / (nx * ny * nz)
    safe = torch.where(k2 == 0, torch.ones_like(k2), k2)
    op = torch.where(k2 == 0, torch.zeros_like(k2), pref * window * torch.exp(-(k2 * rs * rs)) / safe)
    psi = op * rk
    grids = []
    for g in (gx[:, None, None], gy[None, :, None], gz[None, None, :]):
        spec = -1j * g * psi
        grids.append(torch.fft.irfftn(spec, s=(nx, ny, nz), norm="forward"))
    return interpolate(grids, pos, mesh, box, scheme)


def long_inv_r3(r, rs):
    q = 0.5 * r / rs
    t = q * q
    series = (0.125 / rs ** 3) * 4.0 * SQRT_PI_INV * (
        1 / 3 + t * (-1 / 5 + t * (1 / 14 + t * (-1 / 54 + t * (1 / 264 + t * (-1 / 1560 + t * (1 / 10800 - t / 85680)))))))
    full = (torch.erf(q) - 2.0 * SQRT_PI_INV * q * torch.exp(-q * q)) / (r * r * r)
    return torch.where(q < 0.125, series, full)


def neighbor_pairs(pos, box, cutoff):
    """Ordered pairs (i, j), i != j, with min-image distance <= cutoff, from
    detached positions (the pair set is piecewise constant in the positions)."""
    with torch.no_grad():
        p = torch.stack([v.detach() for v in pos], dim=1)
        n = p.shape[0]
        L = torch.tensor(box, dtype=torch.float64, device=p.device)
        ii, jj = [], []
        chunk = max(1, (1 << 24) // max(n, 1))
        for s in range(0, n, chunk):
            d = p[None, :, :] - p[s:s + chunk, None, :]
            d = d - L * torch.round(d / L)
            r2 = (d * d).sum(-1)
            mask = r2 <= cutoff * cutoff
            idx = torch.arange(s, min(s + chunk, n), device=p.device)
            mask[torch.arange(mask.shape[0], device=p.device), idx] = False
            a, b = torch.nonzero(mask, as_tuple=True)
            ii.append(a + s)
            jj.append(b)
        return torch.cat(ii), torch.cat(jj)


def tree_accel(pos, mass, box, rs, cutoff, G, eps, pairs):
    i, j = pairs
    L = [float(v) for v in box]
    d = []
    for a in range(3):
        da = pos[a][j] - pos[a][i]
        d.append(da - L[a] * torch.round(da.detach() / L[a]))
    r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2]
    r = torch.sqrt(r2)
    s2 = r2 + eps * eps
    k = 1.0 / (s2 * torch.sqrt(s2)) - long_inv_r3(r, rs)
    f = G * mass[j] * k
    n = pos[0].shape[0]
    return [torch.zeros(n, dtype=torch.float64, device=pos[0].device).index_add(0, i, f * d[a]) for a in range(3)]


class Problem:
    def __init__(self, mesh, box, G=1.0, asmth_cells=1.25, rcut_cells=6.25, eps=0.0, scheme=0, deconv=True):
        self.mesh, self.box, self.G, self.eps, self.scheme, self.deconv = mesh, box, G, eps, scheme, deconv
        spacing = (box[0] / mesh[0] * box[1] / mesh[1] * box[2] / mesh[2]) ** (1.0 / 3.0)
        self.rs = asmth_cells * spacing
        self.cutoff = rcut_cells * spacing

    def accel(self, pos, mass):
        pairs = neighbor_pairs(pos, self.box, self.cutoff)
        a_pm = pm_accel(pos, mass, self.mesh, self.box, self.rs, self.G, self.scheme, self.deconv)
        a_t = tree_accel(pos, mass, self.box, self.rs, self.cutoff, self.G, self.eps, pairs)
        return [a_pm[k] + a_t[k] for k in range(3)]

    def kdk(self, pos, vel, mass, steps, dt):
        D, K = dt, 0.5 * dt
        L = self.box
        x = list(pos)
        v = list(vel)
        a = self.accel(x, mass)
        for _ in range(steps):
            v = [v[k] + K * a[k] for k in range(3)]
            x = [_canonical(x[k] + D * v[k], L[k]) for k in range(3)]
            a = self.accel(x, mass)
            v = [v[k] + K * a[k] for k in range(3)]
        return x, v


def _canonical(v, L):
    # derivative 1 almost everywhere: subtract the detached number of periods
    return v - L * torch.floor(v.detach() / L)
