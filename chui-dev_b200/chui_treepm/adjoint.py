"""Differentiable TreePM: reverse-mode gradients through KDK steps.

The forward pass runs the library's own kernels (TreePM force, kick, drift)
and keeps one checkpoint of the positions per step. The backward pass walks
the steps in reverse and calls the hand-written adjoint kernels of the C-ABI:

- chui_treepm_force_vjp: x_bar = J_a(x)^T a_bar for the full TreePM
  acceleration at checkpointed positions. PM part: transpose of the force
  interpolation (cotangent deposit plus interpolation-weight gradients), the
  k-space operator transposed (each gradient operator -i k_b G(k) is real and
  odd, so its transpose is its negative), and the transpose of the mass
  deposit (deposit-weight gradients). Short-range part: a walk over the tree
  rebuilt for those positions (interaction lists are recomputed, not stored)
  that evaluates, per pair inside r_cut, G M(d) (m_k a_bar_j - m_j a_bar_k)
  with M(d) = K(r) I + K'(r)/r d d^T, the symmetric form of the pair-force
  Jacobian. Strict-policy multipoles are differentiated as the pairs they
  stand for (exact when no node is accepted, as in lattice-like boxes).
- chui_treepm_kdk_adjoint: the transpose of one static KDK step.
- chui_pm_density_vjp: transpose of the CIC/TSC density for losses on the
  final density.

The reference (cosmosim) has no adjoint; the forward map is its KDK with the
static factors of CosmologicalTimeline::prepareStep (src/core/time_integration.cpp:429-441).
"""
from __future__ import annotations

import torch

from .solver import TreePmCoordinator, kdk_factors_static


def _f64(t):
    return t.detach().to(torch.float64).contiguous()


class TreePmKdk(torch.autograd.Function):
    """steps static KDK steps of size dt from (x, v); returns (x_N, v_N).

    Forces are reused across steps (the closing kick of step k and the opening
    kick of step k+1 act at the same positions), so a forward of N steps costs
    N + 1 force evaluations and the backward N + 1 force VJPs."""

    @staticmethod
    def forward(ctx, x, y, z, vx, vy, vz, mass, solver: TreePmCoordinator, steps: int, dt: float):
        D, K1, K2, drag1, drag2 = kdk_factors_static(dt)
        px, py, pz = _f64(x).clone(), _f64(y).clone(), _f64(z).clone()
        ux, uy, uz = _f64(vx).clone(), _f64(vy).clone(), _f64(vz).clone()
        m = _f64(mass)
        checkpoints = [(px.clone(), py.clone(), pz.clone())]
        r = solver.solve_active_set(px, py, pz, m)
        ax, ay, az = r["ax"], r["ay"], r["az"]
        for _ in range(steps):
            solver.kick(ux, uy, uz, ax, ay, az, K1, drag1)
            solver.drift(px, py, pz, ux, uy, uz, D)
            checkpoints.append((px.clone(), py.clone(), pz.clone()))
            r = solver.solve_active_set(px, py, pz, m)
            ax, ay, az = r["ax"], r["ay"], r["az"]
            solver.kick(ux, uy, uz, ax, ay, az, K2, drag2)
        ctx.solver = solver
        ctx.factors = (D, K1, K2, drag1, drag2)
        ctx.checkpoints = checkpoints
        ctx.save_for_backward(m)
        return px, py, pz, ux, uy, uz

    @staticmethod
    def backward(ctx, gx, gy, gz, gvx, gvy, gvz):
        (m,) = ctx.saved_tensors
        solver: TreePmCoordinator = ctx.solver
        D, K1, K2, drag1, drag2 = ctx.factors
        cps = ctx.checkpoints
        like = cps[0][0]

        def cot(g):
            return torch.zeros_like(like) if g is None else _f64(g).clone()

        xb, yb, zb = cot(gx), cot(gy), cot(gz)
        vxb, vyb, vzb = cot(gvx), cot(gvy), cot(gvz)
        # pending force cotangent at x_N: the closing kick of the last step
        abx, aby, abz = K2 * vxb, K2 * vyb, K2 * vzb
        for k in range(len(cps) - 2, -1, -1):
            px, py, pz = cps[k + 1]
            fx, fy, fz = solver.force_vjp(px, py, pz, m, abx, aby, abz)
            solver.kdk_adjoint(fx, fy, fz, xb, yb, zb, vxb, vyb, vzb, abx, aby, abz,
                               D, K1, K2, drag1, drag2, first_step=(k == 0))
        px, py, pz = cps[0]
        fx, fy, fz = solver.force_vjp(px, py, pz, m, abx, aby, abz)
        xb += fx
        yb += fy
        zb += fz
        ctx.checkpoints = None
        return xb, yb, zb, vxb, vyb, vzb, None, None, None, None


class CicDensity(torch.autograd.Function):
    """Periodic CIC/TSC density (mass / cell volume) on the solver's mesh,
    shape (nx, ny, nz), differentiable with respect to the positions."""

    @staticmethod
    def forward(ctx, x, y, z, mass, solver: TreePmCoordinator):
        px, py, pz, m = _f64(x), _f64(y), _f64(z), _f64(mass)
        rho = solver.assign_density(px, py, pz, m)
        c = solver.config
        ctx.solver = solver
        ctx.save_for_backward(px, py, pz, m)
        return rho.reshape(c.pm_grid_nx, c.pm_grid_ny, c.pm_grid_nz)

    @staticmethod
    def backward(ctx, grho):
        px, py, pz, m = ctx.saved_tensors
        gx, gy, gz = ctx.solver.density_vjp(px, py, pz, m, _f64(grho).reshape(-1))
        return gx, gy, gz, None, None


def kdk(solver: TreePmCoordinator, x, y, z, vx, vy, vz, mass, steps: int, dt: float):
    """Differentiable static KDK integration (see TreePmKdk)."""
    return TreePmKdk.apply(x, y, z, vx, vy, vz, mass, solver, steps, dt)


def cic_density(solver: TreePmCoordinator, x, y, z, mass):
    """Differentiable density on the solver's PM mesh (see CicDensity)."""
    return CicDensity.apply(x, y, z, mass, solver)
