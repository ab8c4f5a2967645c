"""Adjoint kernels (chui_treepm_force_vjp, chui_pm_density_vjp,
chui_treepm_kdk_adjoint) behind the torch.autograd.Functions of
chui_treepm.adjoint, checked against:
- torch autograd through an independent FP64 formulation of the same forward
  map (tests/treepm_torch_reference.py, itself pinned to the C oracle), for
  single VJPs and for the gradient of a density loss after 10 KDK steps on a
  16^3 box (the direct-sum reference gradient);
- central finite differences of the library's own FP64 forward on random
  components of the initial displacements (h = 1e-4 lattice spacing);
- the FP64 adjoint, for the mixed-precision adjoint.
"""
import math

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import chui_treepm as ct  # noqa: E402
from chui_treepm import adjoint, ics  # noqa: E402
import treepm_torch_reference as tr  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dev():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)


def lattice_problem(n_side, box, seed, rms=0.3):
    """Lattice q, Zel'dovich displacement s (P(k) ~ k^-2), unit mean density."""
    x, y, z, sx, sy, sz = ics.zeldovich_lattice(n_side, box, rms, seed)
    spacing = box / n_side
    g = (np.arange(n_side) + 0.5) * spacing
    qx, qy, qz = (a.ravel() for a in np.meshgrid(g, g, g, indexing="ij"))
    m = np.full(n_side ** 3, box ** 3 / n_side ** 3)
    return (qx, qy, qz), (sx, sy, sz), m


def make_solver(n_side, box, precision, mesh=None, eps=0.0, scheme=ct._abi.CIC):
    mesh = mesh or n_side
    return ct.TreePmCoordinator(ct.TreePmConfig(
        pm_grid_nx=mesh, pm_grid_ny=mesh, pm_grid_nz=mesh, box_x=box, box_y=box, box_z=box,
        opening_theta=0.5, max_leaf_size=16, softening=eps, assignment_scheme=scheme, window_deconvolution=1,
        precision=precision))


def rel(a, b):
    a = np.concatenate([np.asarray(v) for v in a])
    b = np.concatenate([np.asarray(v) for v in b])
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("scheme,eps", [(ct._abi.CIC, 0.0), (ct._abi.TSC, 0.05)])
def test_force_vjp_matches_torch_autograd(dev, scheme, eps):
    n_side, box = 16, 12.5
    (qx, qy, qz), (sx, sy, sz), m = lattice_problem(n_side, box, 3)
    pos = [torch.tensor(q + s, device=dev) for q, s in ((qx, sx), (qy, sy), (qz, sz))]
    mass = torch.tensor(m, device=dev)
    rng = np.random.default_rng(9)
    cot = [torch.tensor(rng.normal(size=len(m)), device=dev) for _ in range(3)]

    prob = tr.Problem((n_side,) * 3, (box,) * 3, eps=eps, scheme=scheme, deconv=True)
    p = [v.clone().requires_grad_(True) for v in pos]
    a = prob.accel(p, mass)
    s = sum((a[k] * cot[k]).sum() for k in range(3))
    want = torch.autograd.grad(s, p)
    want = [w.cpu().numpy() for w in want]

    with make_solver(n_side, box, ct._abi.FP64, eps=eps, scheme=scheme) as solver:
        got = solver.force_vjp(*pos, mass, *cot)
        assert solver.last_vjp_stats["kernel_launches"] > 0
    assert rel([g.cpu().numpy() for g in got], want) <= 1e-9

    with make_solver(n_side, box, ct._abi.MIXED, eps=eps, scheme=scheme) as solver:
        got32 = solver.force_vjp(*pos, mass, *cot)
    assert rel([g.cpu().numpy() for g in got32], want) <= 1e-4


def test_density_vjp_matches_torch_autograd(dev):
    n_side, box = 16, 12.5
    (qx, qy, qz), (sx, sy, sz), m = lattice_problem(n_side, box, 4)
    pos = [torch.tensor(q + s, device=dev) for q, s in ((qx, sx), (qy, sy), (qz, sz))]
    mass = torch.tensor(m, device=dev)
    rng = np.random.default_rng(2)
    rho_bar = torch.tensor(rng.normal(size=(n_side,) * 3), device=dev)
    for scheme in (0, 1):
        p = [v.clone().requires_grad_(True) for v in pos]
        rho = tr.deposit(p, mass, (n_side,) * 3, (box,) * 3, scheme)
        want = torch.autograd.grad((rho * rho_bar).sum(), p)
        with make_solver(n_side, box, ct._abi.FP64, scheme=scheme) as solver:
            got = solver.density_vjp(*pos, mass, rho_bar.reshape(-1))
            dens = solver.assign_density(*pos, mass)
        np.testing.assert_allclose(dens.cpu().numpy(), rho.detach().reshape(-1).cpu().numpy(), rtol=1e-12,
                                   atol=1e-12 * rho.abs().max().item())
        assert rel([g.cpu().numpy() for g in got], [w.cpu().numpy() for w in want]) <= 1e-12


def density_loss(solver, dens_solver, q, s, mass, target, steps, dt, vel_factor=1.0):
    x0 = [q[k] + s[k] for k in range(3)]
    v0 = [vel_factor * s[k] for k in range(3)]
    xn = adjoint.kdk(solver, *x0, *v0, mass, steps, dt)
    rho = adjoint.cic_density(dens_solver, xn[0], xn[1], xn[2], mass)
    return ((rho - target) ** 2).mean()


def test_kdk_gradient_matches_direct_sum_reference(dev):
    """16^3 box, 10 KDK steps, loss = MSE(CIC density, target): the library's
    FP64 adjoint against torch autograd through the FP64 direct-sum reference."""
    n_side, box, steps, dt = 16, 12.5, 10, 0.1
    q, s_np, m = lattice_problem(n_side, box, 5)
    q = [torch.tensor(v, device=dev) for v in q]
    mass = torch.tensor(m, device=dev)
    _, s2, _ = lattice_problem(n_side, box, 6)
    with make_solver(n_side, box, ct._abi.FP64) as dsol:
        target = dsol.assign_density(*[q[k] + torch.tensor(s2[k], device=dev) for k in range(3)],
                                     mass).reshape((n_side,) * 3)

    s = [torch.tensor(v, device=dev, requires_grad=True) for v in s_np]
    with make_solver(n_side, box, ct._abi.FP64) as solver, make_solver(n_side, box, ct._abi.FP64) as dsol:
        loss = density_loss(solver, dsol, q, s, mass, target, steps, dt)
        got = torch.autograd.grad(loss, s)

    prob = tr.Problem((n_side,) * 3, (box,) * 3)
    sr = [torch.tensor(v, device=dev, requires_grad=True) for v in s_np]
    x0 = [q[k] + sr[k] for k in range(3)]
    xn, _ = prob.kdk(x0, [sr[k] for k in range(3)], mass, steps, dt)
    rho = tr.deposit(xn, mass, (n_side,) * 3, (box,) * 3, 0)
    loss_ref = ((rho - target) ** 2).mean()
    want = torch.autograd.grad(loss_ref, sr)
    assert abs(loss.item() - loss_ref.item()) <= 1e-9 * abs(loss_ref.item())
    assert rel([g.cpu().numpy() for g in got], [w.cpu().numpy() for w in want]) <= 1e-7


def test_kdk_gradient_matches_finite_differences(dev):
    """64^3 box of 50 (the differentiable benchmark case), 10 KDK steps of
    0.05 at unit mean density with softening 0.1 spacing (unsoftened close
    encounters make the trajectory chaotic, and no gradient check is then
    meaningful): FP64 adjoint gradient vs central differences of the FP64
    forward (deterministic) on 64 random components; mixed adjoint vs FP64
    adjoint.

    With h = 1e-4 spacing the differences straddle the forward map's jumps:
    the residual pair force is cut off at r_cut, where it is ~2.5e-4 of the
    Newtonian force, and CIC weights have kinks at cell faces, so those
    components are compared against the gradient's scale (its largest
    component over all particles). With h = 1e-6 spacing no interval contains
    a jump here, and every component must match on its own."""
    n_side, box, steps, dt = 64, 50.0, 10, 0.05
    spacing = box / n_side
    eps = 0.1 * spacing
    q, s_np, m = lattice_problem(n_side, box, 11)
    q = [torch.tensor(v, device=dev) for v in q]
    mass = torch.tensor(m, device=dev)
    _, s2, _ = lattice_problem(n_side, box, 12)
    with make_solver(n_side, box, ct._abi.FP64) as dsol:
        target = dsol.assign_density(*[q[k] + torch.tensor(s2[k], device=dev) for k in range(3)],
                                     mass).reshape((n_side,) * 3)
    grads = {}
    for prec in (ct._abi.FP64, ct._abi.MIXED):
        s = [torch.tensor(v, device=dev, requires_grad=True) for v in s_np]
        with make_solver(n_side, box, prec, eps=eps) as solver, make_solver(n_side, box, ct._abi.FP64) as dsol:
            loss = density_loss(solver, dsol, q, s, mass, target, steps, dt)
            grads[prec] = [g.cpu().numpy() for g in torch.autograd.grad(loss, s)]
    g64 = grads[ct._abi.FP64]
    assert rel(grads[ct._abi.MIXED], g64) <= 1e-3
    scale = max(float(np.abs(g).max()) for g in g64)
    assert math.isfinite(scale) and scale > 0

    rng = np.random.default_rng(13)
    comps = [(int(rng.integers(3)), int(rng.integers(len(m)))) for _ in range(64)]

    def central(solver, dsol, axis, i, step):
        vals = []
        for sign in (1.0, -1.0):
            s = [torch.tensor(v, device=dev) for v in s_np]
            s[axis][i] += sign * step
            with torch.no_grad():
                vals.append(density_loss(solver, dsol, q, s, mass, target, steps, dt).item())
        return (vals[0] - vals[1]) / (2 * step)

    fd4, fd6, ad = [], [], []
    with make_solver(n_side, box, ct._abi.FP64, eps=eps) as solver, \
            make_solver(n_side, box, ct._abi.FP64) as dsol:
        for axis, i in comps:
            fd4.append(central(solver, dsol, axis, i, 1e-4 * spacing))
            fd6.append(central(solver, dsol, axis, i, 1e-6 * spacing))
            ad.append(g64[axis][i])
    fd4, fd6, ad = np.array(fd4), np.array(fd6), np.array(ad)
    err4 = np.abs(fd4 - ad) / scale
    assert np.median(err4) <= 1e-4 and err4.max() <= 1e-3, (np.median(err4), err4.max())
    err6 = np.abs(fd6 - ad) / np.maximum(np.abs(ad), 1e-3 * scale)
    assert np.median(err6) <= 1e-4 and err6.max() <= 1e-3, (np.median(err6), err6.max())
