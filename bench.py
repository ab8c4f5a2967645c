#!/usr/bin/env python
"""TreePM benchmark: particle-forces/s of the mixed-precision TreePM on one B200,
next to the same solver in FP64 on the GPU and the reference's CPU TreePM.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--workload NAME]

Workload (default "clustered256"): 256^3 = 16,777,216 equal-mass particles in a
periodic box of 200 Mpc/h; 50% in 2000 NFW halos (log-uniform masses over 3
decades, concentrations U[4,12], R_vir ~ M^(1/3)), the rest a Zel'dovich-displaced
lattice (0.5 spacing rms, P(k) ~ k^-2); PM mesh 256^3, r_s = 1.25 cells,
r_cut = 6.25 cells, theta = 0.6, leaf 16, CIC with window deconvolution,
Plummer epsilon 1 kpc/h, strict reference acceptance. Synthetic, seeded inputs
stand in for the reference's external HDF5 initial conditions.

A step is one KDK step: kick with the previous force, drift + periodic wrap,
one full TreePM force evaluation (PM refresh, tree build, residual walk), kick.
`value` counts particle forces (N per step) over the device-timed region with
inputs resident in HBM; `e2e` times the public C-ABI call with host buffers
(pinned), host<->device copies inside the region. Positions (400 MB) exceed L2
(126 MB), so no flush is needed between steps.

Under torchrun with N > 1 every rank runs an independent replica (weak
scaling), timing is the max over ranks. `--shard` instead runs one simulation
across the ranks (strong scaling): every rank holds all particles, walks a
cost-balanced slice of the targets, and one NCCL all-gather per force shares
the accelerations (chui_treepm.sharded).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "chui-dev_b200"))

import numpy as np  # noqa: E402

WORKLOADS = {
    "clustered256": dict(n_side=256, box=200.0, halo_fraction=0.5, n_halos=2000, mass_decades=3.0,
                         lattice_rms=0.5, mesh=256, theta=0.6, leaf=16, eps=0.001),
    "clustered512": dict(n_side=512, box=500.0, halo_fraction=0.6, n_halos=20000, mass_decades=4.0,
                         lattice_rms=0.5, mesh=512, theta=0.7, leaf=32, eps=0.001),
    "clustered128": dict(n_side=128, box=100.0, halo_fraction=0.4, n_halos=300, mass_decades=3.0,
                         lattice_rms=0.5, mesh=128, theta=0.5, leaf=16, eps=0.001),
    "lattice32": dict(n_side=32, box=10.0, halo_fraction=0.0, n_halos=0, mass_decades=0.0,
                      lattice_rms=0.2, mesh=64, theta=0.5, leaf=16, eps=0.0),
}
METRIC = "particle-forces/s at 256^3 (mixed precision TreePM, one KDK step per step)"
UNIT = "particle-forces/s"
# Algorithmic FLOP convention of the walk (fixed, independent of how a kernel
# evaluates the kernel function): 28 per direct pair (3 sub, r^2 5, +eps^2 1,
# rsqrt 1, r^-3 2, residual ~10, accumulate 6), 90 per accepted multipole
# (screened quadrupole), 12 per node visit. Counts are the reference's
# traversal counters for the timed state (the FP64 walk reproduces them).
FLOPS_PER_PAIR = 28.0
FLOPS_PER_MULTIPOLE = 90.0
FLOPS_PER_VISIT = 12.0
# DRAM bytes of one production walk launch on the workload (ncu
# dram__bytes_read.sum + dram__bytes_write.sum, one capture of
# `bench.py --mode profile --workload clustered256`, second walkFast launch)
WALK_DRAM_BYTES = {"clustered256": 11676495872 + 2522083072}
# The differentiable case: 64^3 lattice + Zel'dovich (P ~ k^-2, 0.3 spacing
# rms) in a box of 50, mesh 64^3, theta 0.5, 10 KDK steps of 0.05 at unit mean
# density (G = 1), softening 0.1 spacing, loss = MSE(CIC density of the final
# positions, target).
ADJOINT = dict(n_side=64, box=50.0, steps=10, dt=0.05, theta=0.5, eps_spacing=0.1)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_particles(w: dict, seed: int):
    from chui_treepm import ics
    n = w["n_side"] ** 3
    if w["n_halos"] == 0:
        x, y, z, vx, vy, vz = ics.zeldovich_lattice(w["n_side"], w["box"], w["lattice_rms"], seed)
    else:
        x, y, z, vx, vy, vz = ics.clustered_box(n, w["box"], w["halo_fraction"], w["n_halos"],
                                                w["mass_decades"], w["lattice_rms"], seed)
    m = np.full(n, 1.0 / n)
    return x, y, z, m, vx, vy, vz


def make_config(w: dict, precision: int, device: int, diagnostics: int = 1):
    import chui_treepm as ct
    return ct.TreePmConfig(pm_grid_nx=w["mesh"], pm_grid_ny=w["mesh"], pm_grid_nz=w["mesh"], box_x=w["box"],
                           box_y=w["box"], box_z=w["box"], asmth_cells=1.25, rcut_cells=6.25,
                           opening_theta=w["theta"], max_leaf_size=w["leaf"], assignment_scheme=ct._abi.CIC,
                           window_deconvolution=1, gravitational_constant=1.0, softening=w["eps"],
                           precision=precision, device=device, diagnostics=diagnostics)


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.lines: list[str] = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for name, val in zip(names, parts[3:7]):
                if val.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def rel_errors(a, b):
    num = np.sqrt((a[0] - b[0]) ** 2 + (a[1] - b[1]) ** 2 + (a[2] - b[2]) ** 2)
    den = np.sqrt(b[0] ** 2 + b[1] ** 2 + b[2] ** 2)
    return num / np.maximum(den, 1e-300)


def error_summary(e) -> dict:
    return {"median_rel": float(np.median(e)), "p99_rel": float(np.percentile(e, 99)), "max_rel": float(np.max(e))}


def error_map(err, a_ref, x, y, z, box, cells=64) -> dict:
    """The force-error map of the headline state: the mixed-vs-FP64 relative
    error binned by the FP64 force magnitude (deciles) and by the local number
    density (particles per cell of a 64^3 grid over the mean, by decade)."""
    amag = np.sqrt((a_ref ** 2).sum(axis=0))
    edges = np.quantile(amag, np.linspace(0.0, 1.0, 11))
    by_a = []
    for lo, hi in zip(edges[:-1], edges[1:]):
        sel = (amag >= lo) & (amag <= hi)
        by_a.append({"a_min": float(lo), "a_max": float(hi), "n": int(sel.sum()), **error_summary(err[sel])})
    idx = [np.minimum((np.asarray(c) / box * cells).astype(np.int64), cells - 1) for c in (x, y, z)]
    flat = (idx[0] * cells + idx[1]) * cells + idx[2]
    counts = np.bincount(flat, minlength=cells ** 3)
    dens = counts[flat] / (len(x) / cells ** 3)
    by_rho = []
    for lo, hi in ((0.0, 0.1), (0.1, 1.0), (1.0, 10.0), (10.0, 100.0), (100.0, np.inf)):
        sel = (dens >= lo) & (dens < hi)
        if sel.any():
            by_rho.append({"overdensity_min": lo, "overdensity_max": None if np.isinf(hi) else hi,
                           "n": int(sel.sum()), **error_summary(err[sel])})
    return {"by_force_decile": by_a, "by_local_density": by_rho,
            "density_grid": f"{cells}^3 cells, particle count over the mean"}


def ewald_accuracy(ct, device: int) -> dict:
    """GPU TreePM forces (production mixed walk and FP64) against the direct
    FP64 Ewald sums stored with the reference's outputs in tests/golden (the
    32^3 configuration and the 64000-particle clustered box with the headline
    settings), next to the reference TreePM's own error on the same targets."""
    out = {}
    for name in ("config32", "clustered64k_cic"):
        path = os.path.join(ROOT, "tests", "golden", name + ".npz")
        if not os.path.isfile(path):
            continue
        g = dict(np.load(path))
        k = len(g["ewald_ax"])
        ew = np.stack([g["ewald_ax"], g["ewald_ay"], g["ewald_az"]])
        asmth, rcut, theta, gconst, eps = (float(v) for v in g["params"])
        leaf, scheme, deconv, criterion, order = (int(v) for v in g["iparams"])
        mesh = [int(v) for v in g["mesh"]]
        rec = {"targets": k, "reference_rel_l2": float(np.linalg.norm(
            np.stack([g["ax"][:k], g["ay"][:k], g["az"][:k]]) - ew) / np.linalg.norm(ew))}
        for label, precision, diag in (("mixed_production", ct._abi.MIXED, 0), ("fp64", ct._abi.FP64, 1)):
            cfg = ct.TreePmConfig(pm_grid_nx=mesh[0], pm_grid_ny=mesh[1], pm_grid_nz=mesh[2], box_x=float(g["box"][0]),
                                  box_y=float(g["box"][1]), box_z=float(g["box"][2]), asmth_cells=asmth,
                                  rcut_cells=rcut, opening_theta=theta, opening_criterion=criterion,
                                  multipole_order=order, max_leaf_size=leaf, assignment_scheme=scheme,
                                  window_deconvolution=deconv, gravitational_constant=gconst, softening=eps,
                                  precision=precision, device=device, diagnostics=diag)
            with ct.TreePmCoordinator(cfg) as s:
                r = s.solve_active_set(g["x"], g["y"], g["z"], g["m"])
            got = np.stack([r["ax"][:k], r["ay"][:k], r["az"][:k]])
            per = np.linalg.norm(got - ew, axis=0) / np.linalg.norm(ew, axis=0)
            rec[label] = {"rel_l2": float(np.linalg.norm(got - ew) / np.linalg.norm(ew)),
                          "median_rel": float(np.median(per)), "max_rel": float(per.max())}
        out[name] = rec
    return out


def bench_config(args, w, n, world) -> dict:
    """The workload description both arms print (the same for the reference arm)."""
    return {"workload": f"{args.workload}: N={n}, L={w['box']} Mpc/h, mesh {w['mesh']}^3, "
                        f"r_s=1.25 cells, r_cut=6.25 cells, theta={w['theta']}, leaf {w['leaf']}, "
                        f"CIC+deconvolution, eps={w['eps']}",
            "particles": n, "l2": "inputs larger than L2 (positions 400 MB)",
            "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"}


def gpu_step(solver, t, acc, factors, stream):
    d, k1, k2, g1, g2 = factors
    solver.kick(t["vx"], t["vy"], t["vz"], acc["ax"], acc["ay"], acc["az"], k1, g1, stream=stream)
    solver.drift(t["x"], t["y"], t["z"], t["vx"], t["vy"], t["vz"], d, stream=stream)
    r = solver.solve_active_set(t["x"], t["y"], t["z"], t["m"], stream=stream)
    solver.kick(t["vx"], t["vy"], t["vz"], r["ax"], r["ay"], r["az"], k2, g2, stream=stream)
    return r


def adjoint_bench(torch, ct, dev, local: int) -> dict:
    """Forward (10 KDK steps with one checkpoint per step, then the density
    loss) and backward (the gradient with respect to the initial
    displacements) through chui_treepm.adjoint, timed with CUDA events."""
    from chui_treepm import adjoint, ics
    a = ADJOINT
    n_side, box = a["n_side"], a["box"]
    spacing = box / n_side
    g = (np.arange(n_side) + 0.5) * spacing
    q = [torch.tensor(v.ravel(), device=dev) for v in np.meshgrid(g, g, g, indexing="ij")]
    _, _, _, sx, sy, sz = ics.zeldovich_lattice(n_side, box, 0.3, 101)
    _, _, _, tx, ty, tz = ics.zeldovich_lattice(n_side, box, 0.3, 202)
    mass = torch.full((n_side ** 3,), box ** 3 / n_side ** 3, dtype=torch.float64, device=dev)

    def cfg(precision):
        return ct.TreePmConfig(pm_grid_nx=n_side, pm_grid_ny=n_side, pm_grid_nz=n_side, box_x=box, box_y=box,
                               box_z=box, opening_theta=a["theta"], max_leaf_size=16,
                               softening=a["eps_spacing"] * spacing,
                               assignment_scheme=ct._abi.CIC, window_deconvolution=1, precision=precision,
                               device=local, diagnostics=0)

    with ct.TreePmCoordinator(cfg(ct._abi.MIXED)) as solver, ct.TreePmCoordinator(cfg(ct._abi.MIXED)) as dens:
        target = dens.assign_density(*[q[k] + torch.tensor(v, device=dev) for k, v in enumerate((tx, ty, tz))],
                                     mass).reshape(n_side, n_side, n_side)
        times = []
        for _ in range(3):
            s = [torch.tensor(v, device=dev, requires_grad=True) for v in (sx, sy, sz)]
            e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            torch.cuda.synchronize()
            e[0].record()
            xn = adjoint.kdk(solver, *[q[k] + s[k] for k in range(3)], *s, mass, a["steps"], a["dt"])
            rho = adjoint.cic_density(dens, xn[0], xn[1], xn[2], mass)
            loss = ((rho - target) ** 2).mean()
            e[1].record()
            loss.backward()
            e[2].record()
            torch.cuda.synchronize()
            times.append((e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2])))
        fwd, bwd = min(t[0] for t in times), min(t[1] for t in times)
    return {"workload": f"{n_side}^3 lattice+ZA, L={box}, mesh {n_side}^3, theta {a['theta']}, "
                        f"eps {a['eps_spacing']} spacing, {a['steps']} KDK steps dt={a['dt']}, "
                        f"loss MSE(CIC density)",
            "forward_ms": fwd, "backward_ms": bwd, "backward_over_forward": bwd / fwd,
            "checkpoints": a["steps"] + 1, "precision": "mixed (FP32 pair/mesh, FP64 positions)"}


def vjp_vs_force(torch, solver, t) -> dict:
    """One force VJP against one force evaluation at the same positions."""
    solver.solve_active_set(t["x"], t["y"], t["z"], t["m"])
    cot = [torch.randn_like(t["x"]) for _ in range(3)]
    solver.force_vjp(t["x"], t["y"], t["z"], t["m"], *cot)
    torch.cuda.synchronize()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    e[0].record()
    solver.solve_active_set(t["x"], t["y"], t["z"], t["m"])
    e[1].record()
    solver.force_vjp(t["x"], t["y"], t["z"], t["m"], *cot)
    e[2].record()
    torch.cuda.synchronize()
    f, b = e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2])
    st = solver.last_vjp_stats
    return {"force_ms": f, "vjp_ms": b, "vjp_over_force": b / f,
            "vjp_phases_ms": {k: st[k] for k in ("pm_ms", "tree_build_ms", "walk_ms", "total_ms")}}


def max_over_ranks(torch, dist, value: float, device) -> float:
    """The largest value over all ranks (the job's time is its slowest rank's)."""
    if dist is None:
        return value
    tt = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def timed_steps(torch, solver, t, acc, factors, steps, warmup, dist=None):
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(warmup):
        acc = gpu_step(solver, t, acc, factors, stream)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    launches = 0
    walk_ms = []
    stats = []
    e0.record()
    for _ in range(steps):
        acc = gpu_step(solver, t, acc, factors, stream)
        st = solver.last_stats
        stats.append(st)
        walk_ms.append(st["walk_ms"])
        launches += st["kernel_launches"] + 3  # + kick, drift, kick
    e1.record()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    return e0.elapsed_time(e1), acc, stats, launches


def apply_fast_deck(ct, cfg, group=False):
    """The reference's production fast deck: adaptive relative monopole,
    COM-distance cutoff nodes, alpha 0.0025, maximum angle 1.0 (optionally
    the group walk with the Gaussian pair table)."""
    cfg.acceptance_policy = ct._abi.POLICY_ADAPTIVE
    cfg.adaptive_error_estimator = ct._abi.ESTIMATOR_RELATIVE_MONOPOLE
    cfg.cutoff_node_policy = ct._abi.CUTOFF_COM_DISTANCE
    cfg.adaptive_maximum_opening_angle = 1.0
    cfg.relative_force_tolerance = 0.0025
    if group:
        cfg.group_walk_enabled = 1
        cfg.gaussian_pair_lookup = 1
    return cfg


def adaptive_fast_deck(torch, ct, w, device, t, r_ref, repeats=3) -> dict:
    """One force under the adaptive relative policy (the reference's
    configs/treepm_evolved_snapshot_fast deck settings), production walk:
    device time of the solve and its error against the strict FP64 forces."""
    cfg = apply_fast_deck(ct, make_config(w, ct._abi.MIXED, device, diagnostics=0))
    prev = torch.sqrt(r_ref["ax"] ** 2 + r_ref["ay"] ** 2 + r_ref["az"] ** 2)
    n = len(t["x"])
    with ct.TreePmCoordinator(cfg) as s:
        r = s.solve_active_set(t["x"], t["y"], t["z"], t["m"], previous_acceleration=prev)
        total, walk = [], []
        for _ in range(repeats):
            r = s.solve_active_set(t["x"], t["y"], t["z"], t["m"], previous_acceleration=prev)
            total.append(s.last_stats["total_ms"])
            walk.append(s.last_stats["walk_ms"])
    e = rel_errors([r[k].cpu().numpy() for k in ("ax", "ay", "az")],
                   [r_ref[k].cpu().numpy() for k in ("ax", "ay", "az")])
    ms = float(np.median(total))
    return {"deck": "adaptive relative_monopole, cutoff nodes com_distance, alpha 0.0025, max angle 1.0",
            "value": n / (ms * 1e-3), "unit": "particle-forces/s (one force, device time)",
            "force_ms": ms, "walk_ms": float(np.median(walk)),
            "vs_fp64_strict": {"median_rel": float(np.median(e)), "p99_rel": float(np.percentile(e, 99)),
                               "p9999_rel": float(np.percentile(e, 99.99)), "max_rel": float(np.max(e))}}


def run_gpu(args) -> int:
    import torch
    import chui_treepm as ct

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    w = WORKLOADS[args.workload]
    t0 = time.time()
    x, y, z, m, vx, vy, vz = make_particles(w, seed=42 + rank)
    n = len(x)
    log(f"[rank {rank}] particles {n} generated in {time.time() - t0:.1f}s")
    t = {k: torch.tensor(v, device=dev) for k, v in dict(x=x, y=y, z=z, m=m, vx=vx, vy=vy, vz=vz).items()}
    factors = ct.kdk_factors_static(args.dt)

    # production walk (diagnostics off: no per-pair counters, subtree blocks)
    mixed = ct.TreePmCoordinator(make_config(w, ct._abi.MIXED, local, diagnostics=0))
    # the per-node FP64 walk that reproduces the reference's traversal counters
    # (the FLOP convention's counts, the accuracy reference)
    fp64 = ct.TreePmCoordinator(make_config(w, ct._abi.FP64, local, diagnostics=1))

    # accuracy of the production walk against the FP64 walk on the initial state
    r_m = mixed.solve_active_set(t["x"], t["y"], t["z"], t["m"])
    r_d = fp64.solve_active_set(t["x"], t["y"], t["z"], t["m"])
    a_mixed = np.stack([r_m[k].cpu().numpy() for k in ("ax", "ay", "az")])
    a_fp64 = np.stack([r_d[k].cpu().numpy() for k in ("ax", "ay", "az")])
    err = rel_errors(a_mixed, a_fp64)
    err_map = error_map(err, a_fp64, x, y, z, w["box"])
    # the reference's traversal counters (pairs inside r_cut etc.) come from the FP64 walk
    stats0 = dict(fp64.last_stats)
    log(f"[rank {rank}] mixed vs fp64 median {np.median(err):.3e} p99 {np.percentile(err, 99):.3e}; "
        f"stats {stats0}")

    # the reference's production fast deck on the same state: adaptive relative
    # monopole, COM-distance cutoff nodes, alpha 0.0025, maximum angle 1.0, with
    # the FP64 strict solve's |a| as the acceleration history
    adaptive = adaptive_fast_deck(torch, ct, w, local, t, r_d)
    log(f"[rank {rank}] adaptive fast deck {adaptive}")

    fp64.close()
    del r_d
    torch.cuda.empty_cache()
    # FP64-on-GPU comparator: the same production solver (traversal, subtree
    # blocks, tiled deposit) with FP64 pairs, multipoles and mesh; same step
    # definition, fewer repetitions
    fp64p = ct.TreePmCoordinator(make_config(w, ct._abi.FP64, local, diagnostics=0))
    r_p = fp64p.solve_active_set(t["x"], t["y"], t["z"], t["m"])
    a_fp64p = np.stack([r_p[k].cpu().numpy() for k in ("ax", "ay", "az")])
    err_fp64p = rel_errors(a_fp64p, a_fp64)
    tf = {k: v.clone() for k, v in t.items()}
    fp64_ms, _, fp64_stats, _ = timed_steps(torch, fp64p, tf, r_p, factors, max(1, args.fp64_steps), 1)
    fp64_value = n * max(1, args.fp64_steps) / (fp64_ms * 1e-3)
    fp64_phases = {k: fp64_stats[-1][k] for k in ("pm_ms", "tree_build_ms", "walk_ms", "total_ms")}
    del tf, r_p
    fp64p.close()
    torch.cuda.empty_cache()

    # headline: mixed precision, device-resident inputs
    with ClockSampler(local) as clocks:
        ms, acc, stats, launches = timed_steps(torch, mixed, t, r_m, factors, args.steps, args.warmup, dist)
    ms = max_over_ranks(torch, dist, ms, dev)
    value = n * args.steps * world / (ms * 1e-3)

    # end to end through the C-ABI with pinned host buffers: the same KDK step
    # (kick, drift, force, kick), every call staging its host arrays in and
    # its results out
    def pinned(a):
        return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()

    h = {k: pinned(v) for k, v in dict(x=x, y=y, z=z, m=m, vx=vx, vy=vy, vz=vz).items()}
    # the accelerations come back into pinned host arrays the caller keeps
    houts = [pinned(np.zeros(n)) for _ in range(3)]
    mixed.solve_active_set(h["x"], h["y"], h["z"], h["m"], out=houts)  # warm
    e2e_steps = max(1, min(args.steps, 3))
    d_f, k1_f, k2_f, g1_f, g2_f = factors
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    for _ in range(e2e_steps):
        mixed.kick(h["vx"], h["vy"], h["vz"], houts[0], houts[1], houts[2], k1_f, g1_f)
        mixed.drift(h["x"], h["y"], h["z"], h["vx"], h["vy"], h["vz"], d_f)
        mixed.solve_active_set(h["x"], h["y"], h["z"], h["m"], out=houts)
        mixed.kick(h["vx"], h["vy"], h["vz"], houts[0], houts[1], houts[2], k2_f, g2_f)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - w0
    e2e_value = n * e2e_steps * world / max_over_ranks(torch, dist, e2e_s, dev)
    del h, houts

    # roofline of the dominant kernel (residual walk, FP32 pipes)
    peak = ct.probe_fp32_peak_tflops(local)
    st = stats[-1]
    # algorithmic work: the reference's traversal counters for the timed state
    # (the first step's counts; positions move by far less than a leaf per step)
    walk_flops = (FLOPS_PER_PAIR * stats0["direct_pair_evaluations"] +
                  FLOPS_PER_MULTIPOLE * stats0["accepted_internal_multipoles"] +
                  FLOPS_PER_VISIT * stats0["visited_nodes"])
    achieved = walk_flops / (st["walk_ms"] * 1e-3) / 1e12
    checks = mixed.momentum_energy(t["m"], t["vx"], t["vy"], t["vz"], acc["ax"], acc["ay"], acc["az"])
    try:
        adj_step = vjp_vs_force(torch, mixed, t)
    except Exception as exc:  # reported, not fatal to the headline
        adj_step = {"error": repr(exc)}
    mixed.close()
    del t, acc
    torch.cuda.empty_cache()
    try:
        adj = adjoint_bench(torch, ct, dev, local)
        adj["one_step_at_workload"] = adj_step
    except Exception as exc:
        adj = {"error": repr(exc), "one_step_at_workload": adj_step}

    if rank == 0:
        result = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 pair/mesh arithmetic, f64 positions/decisions/COM",
            "data": "synthetic (seeded NFW halos + Zel'dovich lattice)",
            "config": bench_config(args, w, n, world),
            "accuracy_vs_fp64_gpu": {"median_rel": float(np.median(err)),
                                     "p99_rel": float(np.percentile(err, 99)),
                                     "max_rel": float(np.max(err)), "error_map": err_map},
            "fp64_gpu": {"value": fp64_value, "unit": UNIT, "steps": max(1, args.fp64_steps),
                         "solver": "the production solver in FP64: same traversal, subtree blocks and tiled "
                                   "deposit; FP64 pairs (the reference's erf/exp residual), multipoles, mesh and FFT",
                         "phases_ms": fp64_phases,
                         "vs_fp64_counter_exact_walk": error_summary(err_fp64p),
                         "speedup_mixed_over_fp64": value / world / fp64_value},
            "phases_ms": {k: st[k] for k in ("pm_ms", "tree_build_ms", "walk_ms", "total_ms")},
            "counters": {k: stats0[k] for k in ("direct_pair_evaluations", "visited_nodes",
                                                "accepted_internal_multipoles", "node_count", "maximum_depth")},
            "adjoint": adj,
            "adaptive_fast_deck": adaptive,
            "fp64_checks_end": {"momentum": [float(v) for v in checks["momentum"]],
                                "net_force": [float(v) for v in checks["net_force"]],
                                "kinetic_energy": checks["kinetic_energy"], "mass": checks["mass"]},
            "roofline": {"bound": "fp32", "kernel": "walkFastKernel (production walk)", "achieved": achieved,
                         "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                         "peak_source": "measured FP32 FFMA probe (chui_treepm_probe_fp32_peak)",
                         "flops_convention": {"pair": FLOPS_PER_PAIR, "multipole": FLOPS_PER_MULTIPOLE,
                                              "visit": FLOPS_PER_VISIT},
                         "traffic": WALK_DRAM_BYTES.get(args.workload),
                         "traffic_unit": "bytes per launch (ncu dram__bytes_read.sum + dram__bytes_write.sum)"},
            "e2e": {"value": e2e_value, "unit": UNIT,
                    # kick (v, a in; v out), drift (x, v in; x out), force (x, m in; a out), kick
                    "h2d_bytes_per_step": n * (48 + 48 + 32 + 48), "d2h_bytes_per_step": n * (24 + 24 + 24 + 24),
                    "steps": e2e_steps, "step": "one KDK step through the C-ABI with pinned host buffers"},
            "gpu_launches": launches,
            "clocks": clocks.summary(),
        }
        if args.cpu_baseline:
            cb, ref, act = cpu_baseline(w, x, y, z, m, args)
            if cb is not None:
                result["cpu_baseline"] = cb
                a_ref = np.stack([ref["ax"], ref["ay"], ref["az"]])
                result["accuracy_vs_reference"] = {
                    "targets": int(len(act)),
                    "sample": "the reference's own TreePM accelerations at the CPU baseline's seeded targets, "
                              "same initial state and settings",
                    "mixed_production": error_summary(rel_errors(a_mixed[:, act], a_ref)),
                    "fp64_gpu": error_summary(rel_errors(a_fp64[:, act], a_ref)),
                    "fp64_gpu_production": error_summary(rel_errors(a_fp64p[:, act], a_ref)),
                    "reference_vs_fp64_gpu_max_abs_over_max": float(
                        np.abs(a_fp64[:, act] - a_ref).max() / np.abs(a_ref).max())}
        result["accuracy_vs_ewald"] = ewald_accuracy(ct, local)
        print(json.dumps(result), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def sharded_step(sharded, solver, t, acc, factors, stream):
    """One KDK step of one simulation held by every rank: the force's walk is
    split across the ranks, every rank kicks and drifts all particles."""
    d, k1, k2, g1, g2 = factors
    solver.kick(t["vx"], t["vy"], t["vz"], acc[0], acc[1], acc[2], k1, g1, stream=stream)
    solver.drift(t["x"], t["y"], t["z"], t["vx"], t["vy"], t["vz"], d, stream=stream)
    acc = sharded.accelerations(t["x"], t["y"], t["z"], t["m"], stream=stream)
    solver.kick(t["vx"], t["vy"], t["vz"], acc[0], acc[1], acc[2], k2, g2, stream=stream)
    return acc


def run_sharded(args) -> int:
    """--shard: one simulation across the ranks (sources replicated, the walk's
    targets sliced by cost, one all-gather of the accelerations per force;
    chui_treepm.sharded). Strong scaling: the particle count is fixed."""
    import datetime

    import torch
    import chui_treepm as ct

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    w = WORKLOADS[args.workload]
    # the same particles on every rank: one simulation
    x, y, z, m, vx, vy, vz = make_particles(w, seed=42)
    n = len(x)
    t = {k: torch.tensor(v, device=dev) for k, v in dict(x=x, y=y, z=z, m=m, vx=vx, vy=vy, vz=vz).items()}
    factors = ct.kdk_factors_static(args.dt)
    solver = ct.TreePmCoordinator(make_config(w, ct._abi.MIXED, local, diagnostics=0))
    sharded = ct.ShardedTreePm(solver, group=None if dist is not None else False)
    stream = torch.cuda.current_stream().cuda_stream
    acc = sharded.accelerations(t["x"], t["y"], t["z"], t["m"], stream=stream)
    for _ in range(args.warmup):
        acc = sharded_step(sharded, solver, t, acc, factors, stream)
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    launches = 0
    slices = []
    with ClockSampler(local) as clocks:
        e0.record()
        for _ in range(args.steps):
            acc = sharded_step(sharded, solver, t, acc, factors, stream)
            launches += solver.last_stats["kernel_launches"] + 3
            slices.append({"counts": list(sharded.last_counts), "walk_ms": list(sharded.last_walk_ms)})
        e1.record()
        torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    ms = max_over_ranks(torch, dist, e0.elapsed_time(e1), dev)
    value = n * args.steps / (ms * 1e-3)
    st = dict(solver.last_stats)
    solver.close()
    if rank == 0:
        result = {
            "metric": METRIC,
            "value": value,
            "unit": UNIT,
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms / args.steps,
            "higher_is_better": True,
            "scaling": "strong",
            "vs_baseline": None,
            "dtype": "f32 pair/mesh arithmetic, f64 positions/decisions/COM",
            "data": "synthetic (seeded NFW halos + Zel'dovich lattice)",
            "config": {"workload": f"{args.workload}: N={n}, L={w['box']} Mpc/h, mesh {w['mesh']}^3, "
                                   f"theta={w['theta']}, leaf {w['leaf']}",
                       "particles": n, "l2": "inputs larger than L2 (positions 400 MB)",
                       "parallelism": f"shard{world}: sources replicated, walk targets sliced by cost, "
                                      "one all-gather of accelerations per force"},
            "phases_ms_rank0": {k: st[k] for k in ("pm_ms", "tree_build_ms", "walk_ms", "total_ms")},
            "slices_last_step": slices[-1] if slices else None,
            "gpu_launches": launches,
            "clocks": clocks.summary(),
            "e2e": None,
        }
        print(json.dumps(result), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def cpu_baseline(w, x, y, z, m, args, warmup: int = 1, steps: int = 1):
    """The reference's own TreePM (oracle/_ref/treepm_ref, built from its
    sources) on the host cores, all in one process: full PM + tree build, and
    the residual walk on a seeded 1/64 target subset whose traversal time is
    scaled to all N targets. The process's first solve and the next
    warmup - 1 are warm-up; the value is the median of the estimates of the
    following `steps` solves. Returns (summary, reference result, targets),
    or (None, None, None) without the reference build."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refio
    if not refio.available():
        return None, None, None
    n = len(x)
    frac = args.cpu_fraction
    rng = np.random.default_rng(7)
    k = max(1, int(n * frac))
    act = np.sort(rng.choice(n, k, replace=False)).astype(np.uint32)
    warmup = max(1, warmup)
    p = refio.RefProblem(x, y, z, m, box=(w["box"],) * 3, mesh=(w["mesh"],) * 3, theta=w["theta"], leaf=w["leaf"],
                         eps=w["eps"], deconv=1, active=act, dump_tree=0, repeats=warmup - 1 + steps)
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    r = refio.run(p, threads=cores)
    wall = time.perf_counter() - t0
    ph = r["repeat_phases_ms"][warmup - 1:]
    tot = r["repeat_ms"][warmup - 1:]
    # per solve: everything as measured, except the traversal (per target),
    # which is scaled from the k sampled targets to all n
    est = [float(t - trav + trav * n / k) for t, (pm, build, trav) in zip(tot, ph)]
    est_ms = statistics.median(est)
    i = est.index(sorted(est)[len(est) // 2]) if len(est) % 2 else 0
    pm, build, trav = (float(v) for v in ph[i])
    summary = {"value": n / (est_ms * 1e-3), "unit": UNIT, "cores": cores, "kind": "reference",
               "cpu_model": refio.host_cpu(), "build": f"g++ -O3 -fopenmp -march={refio.build_arch()}",
               "warmup": warmup, "steps": steps, "solve_ms_estimates": est,
               "sample": f"one process: {warmup} warm-up + {steps} timed full solves (PM {w['mesh']}^3 with the "
                         f"FFT of the repository's FFTW-API shim, full tree build), residual walk on {k} seeded "
                         f"targets ({frac:.4f} of N) with its traversal time scaled by N/{k}; median of the timed "
                         f"solves",
               "phases_ms": {"pm": pm, "tree_build": build, "walk_sample": trav, "walk_scaled": trav * n / k,
                             "rest": float(tot[i]) - pm - build - trav},
               "process_wall_s": wall}
    return summary, r, act


def run_profile(args) -> int:
    """Two production (mixed precision, diagnostics off) force evaluations of
    the workload (the second is the one an ncu capture selects with -s/-c),
    nothing else: for launch lists and single-kernel captures. --mode
    profile-vjp runs two force VJPs instead. --deck fast / fast-group: the
    adaptive fast deck (per-target / group walk), history from a first
    strict solve."""
    import torch
    import chui_treepm as ct
    w = WORKLOADS[args.workload]
    x, y, z, m, vx, vy, vz = make_particles(w, seed=42)
    dev = torch.device("cuda", 0)
    t = {k: torch.tensor(v, device=dev) for k, v in dict(x=x, y=y, z=z, m=m).items()}
    cfg = make_config(w, ct._abi.FP64 if args.precision == "fp64" else ct._abi.MIXED, 0, diagnostics=0)
    prev = None
    if args.deck != "strict":
        with ct.TreePmCoordinator(cfg) as s:
            r = s.solve_active_set(t["x"], t["y"], t["z"], t["m"])
            prev = torch.sqrt(r["ax"] ** 2 + r["ay"] ** 2 + r["az"] ** 2)
            del r
        apply_fast_deck(ct, cfg, group=args.deck == "fast-group")
    with ct.TreePmCoordinator(cfg) as s:
        if args.mode == "profile-vjp":
            # two force VJPs with seeded Gaussian cotangents (the adjoint's hot call)
            g = torch.Generator(device="cpu").manual_seed(1)
            cot = [torch.randn(len(x), generator=g, dtype=torch.float64).to(dev) for _ in range(3)]
            for _ in range(2):
                s.force_vjp(t["x"], t["y"], t["z"], t["m"], *cot)
            torch.cuda.synchronize()
            log(json.dumps(s.last_vjp_stats))
            return 0
        for _ in range(2):
            s.solve_active_set(t["x"], t["y"], t["z"], t["m"], previous_acceleration=prev)
        torch.cuda.synchronize()
        log(json.dumps(s.last_stats))
    return 0


def run_reference(args) -> int:
    """The reference arm: the reference's CPU TreePM (cpu_baseline) on the
    same workload, one warm-up and a median over timed solves in one process.
    At 256^3 a full solve takes ~20 s on 16 host cores (the tree build and PM
    alone are most of it), so the arm times at most 3 solves after 1 warm-up
    whatever --steps/--warmup ask, to end within a few minutes."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refio
    w = WORKLOADS[args.workload]
    if not refio.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference oracle binary oracle/_ref/treepm_ref "
                                                              "not built (needs the reference sources)"}))
        return 0
    x, y, z, m, vx, vy, vz = make_particles(w, seed=42)
    n = len(x)
    big = args.workload in ("clustered256", "clustered512")
    steps = min(args.steps, 3) if big else args.steps
    warmup = min(max(args.warmup, 1), 1) if big else max(args.warmup, 1)
    cb, _, _ = cpu_baseline(w, x, y, z, m, args, warmup=warmup, steps=steps)
    value = cb["value"]
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0,
        "steps": steps, "warmup": warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded NFW halos + Zel'dovich lattice)",
        "config": bench_config(args, w, n, 1),
        "cpu_baseline": cb,
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)
    return 0


def run_large(args) -> int:
    """The large configuration (default clustered512: 512^3 = 134M particles,
    L = 500, 60 % in 20000 halos over 4 decades, mesh 512^3, theta 0.7, leaf
    32): one production force, the traversal counters (per-node walk), the
    mixed-vs-FP64 force error on a seeded 1/256 target subset, and the adjoint
    of one KDK step (forward, then the gradient of sum(w . x_1) with respect
    to the initial positions). Prints one JSON record (not the headline)."""
    import torch
    import chui_treepm as ct
    from chui_treepm import adjoint
    w = WORKLOADS[args.workload]
    dev = torch.device("cuda", 0)
    t0 = time.time()
    x, y, z, m, vx, vy, vz = make_particles(w, seed=42)
    n = len(x)
    log(f"particles {n} generated in {time.time() - t0:.1f}s")
    t = {k: torch.tensor(v, device=dev) for k, v in dict(x=x, y=y, z=z, m=m, vx=vx, vy=vy, vz=vz).items()}
    del x, y, z, vx, vy, vz
    rec = {"workload": args.workload, "particles": n, "config": w}

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        out = fn()
        e1.record()
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1)

    with ct.TreePmCoordinator(make_config(w, ct._abi.MIXED, 0, diagnostics=0)) as s:
        s.solve_active_set(t["x"], t["y"], t["z"], t["m"])
        r, ms = timed(lambda: s.solve_active_set(t["x"], t["y"], t["z"], t["m"]))
        st = dict(s.last_stats)
        rec["force"] = {"ms": ms, "particle_forces_per_s": n / (ms * 1e-3),
                        "phases_ms": {k: st[k] for k in ("pm_ms", "tree_build_ms", "walk_ms", "total_ms")}}
        rng = np.random.default_rng(7)
        sub = np.sort(rng.choice(n, n // 256, replace=False)).astype(np.uint32)
        mixed_sub = np.stack([r[k].cpu().numpy()[sub] for k in ("ax", "ay", "az")])
        del r
        # PM algorithmic bytes (deposit 24N + 8M, R2C + 3 C2R, Green 32 Mc, interpolation 24N + 12M + 12N)
        mesh = w["mesh"]
        cells = mesh ** 3
        mc = mesh * mesh * (mesh // 2 + 1)
        pm_bytes = (24 * n + 8 * cells) + 4 * (4 * cells + 8 * mc) + 32 * mc
        rec["pm_refresh_effective_gbs"] = pm_bytes / (st["pm_ms"] * 1e-3) / 1e9
    torch.cuda.empty_cache()
    with ct.TreePmCoordinator(make_config(w, ct._abi.MIXED, 0, diagnostics=1)) as s:
        s.solve_active_set(t["x"], t["y"], t["z"], t["m"])
        c = dict(s.last_stats)
        rec["counters"] = {k: c[k] for k in ("direct_pair_evaluations", "visited_nodes",
                                             "accepted_internal_multipoles", "node_count", "maximum_depth")}
        flops = (FLOPS_PER_PAIR * c["direct_pair_evaluations"] + FLOPS_PER_MULTIPOLE *
                 c["accepted_internal_multipoles"] + FLOPS_PER_VISIT * c["visited_nodes"])
        rec["walk_achieved_tflops"] = flops / (rec["force"]["phases_ms"]["walk_ms"] * 1e-3) / 1e12
        rec["walk_fraction_of_fp32_peak"] = rec["walk_achieved_tflops"] / ct.probe_fp32_peak_tflops(0)
    torch.cuda.empty_cache()
    with ct.TreePmCoordinator(make_config(w, ct._abi.FP64, 0, diagnostics=1)) as s:
        sub_t = torch.tensor(sub.astype(np.int64), device=dev)
        r, ms64 = timed(lambda: s.solve_active_set(t["x"], t["y"], t["z"], t["m"], active=sub_t))
        ref = np.stack([r[k].cpu().numpy() for k in ("ax", "ay", "az")])
        e = rel_errors(mixed_sub, ref)
        rec["accuracy_vs_fp64_subset"] = {"targets": int(len(sub)), "median_rel": float(np.median(e)),
                                          "p99_rel": float(np.percentile(e, 99)), "max_rel": float(np.max(e)),
                                          "fp64_subset_ms": ms64}
        del r
    torch.cuda.empty_cache()
    # adjoint of one KDK step
    with ct.TreePmCoordinator(make_config(w, ct._abi.MIXED, 0, diagnostics=0)) as s:
        g = torch.Generator(device="cpu").manual_seed(3)
        wts = [torch.randn(n, generator=g, dtype=torch.float64).to(dev) for _ in range(3)]
        pos = [t[k].clone().requires_grad_(True) for k in ("x", "y", "z")]

        def fwd():
            out = adjoint.kdk(s, *pos, t["vx"], t["vy"], t["vz"], t["m"], 1, args.dt)
            return sum((out[k] * wts[k]).sum() for k in range(3))

        loss, fwd_ms = timed(fwd)
        _, bwd_ms = timed(lambda: loss.backward())
        gnorm = float(sum((p.grad ** 2).sum() for p in pos).sqrt())
        rec["adjoint_one_kdk_step"] = {"forward_ms": fwd_ms, "backward_ms": bwd_ms,
                                       "backward_over_forward": bwd_ms / fwd_ms, "grad_norm": gnorm,
                                       "finite": bool(np.isfinite(gnorm))}
    print(json.dumps(rec), flush=True)
    return 0


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="clustered256", choices=sorted(WORKLOADS))
    ap.add_argument("--dt", type=float, default=1.0e-3)
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--cpu-fraction", type=float, default=1.0 / 64.0)
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--mode", default="bench", choices=["bench", "profile", "profile-vjp", "large"])
    ap.add_argument("--deck", default="strict", choices=["strict", "fast", "fast-group"],
                    help="acceptance settings of --mode profile")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"], help="precision of --mode profile")
    ap.add_argument("--shard", action="store_true",
                    help="one simulation across the ranks (strong scaling) instead of one replica per rank")
    args = ap.parse_args()
    if args.mode in ("profile", "profile-vjp"):
        return run_profile(args)
    if args.mode == "large":
        if args.workload == "clustered256":
            args.workload = "clustered512"
        return run_large(args)
    if args.impl == "reference":
        return run_reference(args)
    if args.shard:
        return run_sharded(args)
    return run_gpu(args)


if __name__ == "__main__":
    sys.exit(main())
