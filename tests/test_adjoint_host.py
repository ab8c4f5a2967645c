"""Host logic of chui_treepm.adjoint on CPU: the reverse sweep of TreePmKdk
(force reuse across steps, combined kick cotangents, one force VJP per
checkpoint) and the transpose-of-KDK formula that chui_treepm_kdk_adjoint
implements, checked with a stand-in solver whose force is analytic, against
torch autograd through the same forward written in plain torch."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from chui_treepm import adjoint  # noqa: E402
from chui_treepm.solver import kdk_factors_static  # noqa: E402


class AnalyticSolver:
    """a = -k x + c sin(x) per component; the methods mirror TreePmCoordinator."""

    k, c = 0.7, 0.3

    def accel(self, x):
        return -self.k * x + self.c * torch.sin(x)

    def solve_active_set(self, x, y, z, m):
        return {"ax": self.accel(x), "ay": self.accel(y), "az": self.accel(z)}

    def kick(self, vx, vy, vz, ax, ay, az, kick, drag):
        for v, a in ((vx, ax), (vy, ay), (vz, az)):
            v.mul_(drag).add_(kick * a)

    def drift(self, x, y, z, vx, vy, vz, d):
        for p, v in ((x, vx), (y, vy), (z, vz)):
            p.add_(d * v)

    def force_vjp(self, x, y, z, m, cx, cy, cz):
        return tuple(c * (-self.k + self.c * torch.cos(p)) for p, c in ((x, cx), (y, cy), (z, cz)))

    def kdk_adjoint(self, gx, gy, gz, xb, yb, zb, vxb, vyb, vzb, axb, ayb, azb, D, K1, K2, drag1, drag2,
                    first_step):
        # the formula of chui_treepm_kdk_adjoint (include/chui_treepm.h)
        for g, xbar, vbar, abar in ((gx, xb, vxb, axb), (gy, yb, vyb, ayb), (gz, zb, vzb, azb)):
            xbar.add_(g)
            vh = drag2 * vbar + D * xbar
            vbar.copy_(drag1 * vh)
            abar.copy_(K1 * vh + (0.0 if first_step else K2) * vbar)


def plain_kdk(solver, x, v, steps, dt):
    D, K1, K2, g1, g2 = kdk_factors_static(dt)
    a = [solver.accel(p) for p in x]
    for _ in range(steps):
        v = [g1 * v[k] + K1 * a[k] for k in range(3)]
        x = [x[k] + D * v[k] for k in range(3)]
        a = [solver.accel(p) for p in x]
        v = [g2 * v[k] + K2 * a[k] for k in range(3)]
    return x, v


@pytest.mark.parametrize("steps", [1, 3, 7])
def test_reverse_sweep_matches_autograd(steps):
    rng = np.random.default_rng(steps)
    n, dt = 50, 0.13
    x0 = [torch.tensor(rng.normal(size=n), requires_grad=True) for _ in range(3)]
    v0 = [torch.tensor(rng.normal(size=n), requires_grad=True) for _ in range(3)]
    wx = [torch.tensor(rng.normal(size=n)) for _ in range(3)]
    wv = [torch.tensor(rng.normal(size=n)) for _ in range(3)]
    m = torch.ones(n, dtype=torch.float64)
    solver = AnalyticSolver()

    out = adjoint.kdk(solver, *x0, *v0, m, steps, dt)
    loss = sum((out[k] * wx[k]).sum() + (out[3 + k] * wv[k]).sum() for k in range(3))
    got = torch.autograd.grad(loss, x0 + v0)

    xr = [t.detach().clone().requires_grad_(True) for t in x0]
    vr = [t.detach().clone().requires_grad_(True) for t in v0]
    xn, vn = plain_kdk(solver, xr, vr, steps, dt)
    loss_ref = sum((xn[k] * wx[k]).sum() + (vn[k] * wv[k]).sum() for k in range(3))
    want = torch.autograd.grad(loss_ref, xr + vr)
    assert abs(loss.item() - loss_ref.item()) <= 1e-12 * abs(loss_ref.item())
    for g, w in zip(got, want):
        np.testing.assert_allclose(g.numpy(), w.numpy(), rtol=1e-12, atol=1e-12)
