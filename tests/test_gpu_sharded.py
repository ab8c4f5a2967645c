"""Target-sharded solves on the GPU (chui_treepm_solve_visit_range,
chui_treepm_visit_order, chui_treepm_walk_cost, chui_treepm.sharded).

The union of the slices of the visit order is the full solve: with the PM
field of the full solve reused, every slice reproduces the full solve's
accelerations of its targets (FP64 to 1e-12 of the largest, the mixed walk to
1e-6), its long-range lanes bit for bit, and the slices' traversal counters
sum to the full solve's. Two processes sharing this GPU (gloo between them;
no kernel of one waits on the other) run three KDK steps of one simulation
through ShardedTreePm and end where the single-process run ends.
"""
import os
import socket
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")

import chui_treepm as ct  # noqa: E402
from chui_treepm import ics, sharded  # noqa: E402

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
N_SIDE, BOX = 32, 10.0
COUNTERS = ("visited_nodes", "accepted_nodes", "opened_nodes", "direct_pair_evaluations", "cutoff_pruned_nodes",
            "cutoff_skipped_pairs", "accepted_internal_multipoles", "accepted_leaves")


@pytest.fixture(scope="module")
def cuda_ok():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True


def _particles(device):
    n = N_SIDE ** 3
    x, y, z, vx, vy, vz = ics.clustered_box(n, BOX, 0.4, 30, 2.0, 0.3, 5)
    m = np.full(n, 1.0 / n)
    return {k: torch.tensor(v, device=device) for k, v in dict(x=x, y=y, z=z, m=m, vx=vx, vy=vy, vz=vz).items()}


def _config(precision, diagnostics=1):
    return ct.TreePmConfig(pm_grid_nx=32, pm_grid_ny=32, pm_grid_nz=32, box_x=BOX, box_y=BOX, box_z=BOX,
                           opening_theta=0.5, max_leaf_size=16, softening=0.002, precision=precision,
                           diagnostics=diagnostics)


@pytest.mark.parametrize("precision,diagnostics", [(ct._abi.FP64, 1), (ct._abi.MIXED, 1), (ct._abi.MIXED, 0)])
@pytest.mark.parametrize("shards", [2, 3])
def test_slices_reassemble_the_full_solve(cuda_ok, precision, diagnostics, shards):
    t = _particles("cuda")
    n = len(t["x"])
    with ct.TreePmCoordinator(_config(precision, diagnostics)) as s:
        full = s.solve_active_set(t["x"], t["y"], t["z"], t["m"], long_range=True)
        full_stats = dict(s.last_stats)
        order = s.visit_order(0, n, device="cuda")
        bounds = sharded.even_bounds(n, shards)
        got = {k: torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
               for k in ("ax", "ay", "az", "pm_ax", "pm_ay", "pm_az")}
        sums = dict.fromkeys(COUNTERS, 0)
        for q in range(shards):
            b, e = bounds[q], bounds[q + 1]
            r = s.solve_active_set_with_pm_cadence(t["x"], t["y"], t["z"], t["m"], False, long_range=True,
                                                   visit_range=(b, e))
            assert torch.equal(s.visit_order(b, e, device="cuda"), order[b:e])
            for k in got:
                assert r[k].numel() == e - b
                got[k][order[b:e]] = r[k]
            for k in COUNTERS:
                sums[k] += r["stats"][k]
            cost = s.walk_cost(0, n)
            inside = cost[b // 32:(e + 31) // 32]
            outside = np.concatenate([cost[: b // 32], cost[(e + 31) // 32:]])
            assert (outside == 0).all()
            # recorded by the FP64 walk and the mixed production walk (no diagnostics)
            recorded = precision == ct._abi.FP64 or not diagnostics
            assert (inside > 0).all() if recorded else (inside == 0).all()
    scale = max(float(full[k].abs().max()) for k in ("ax", "ay", "az"))
    tol = 1e-12 if precision == ct._abi.FP64 else 1e-6
    for k in ("ax", "ay", "az"):
        assert float((got[k] - full[k]).abs().max()) <= tol * scale, k
        assert torch.equal(got["pm_" + k], full["pm_" + k])
    if diagnostics:
        if precision == ct._abi.FP64:
            assert sums == {k: full_stats[k] for k in COUNTERS}
        else:
            # node counters; the FP32 pair-cutoff test may count differently within rounding of r_cut
            node = ("visited_nodes", "accepted_nodes", "opened_nodes", "cutoff_pruned_nodes",
                    "accepted_internal_multipoles", "accepted_leaves")
            assert [sums[k] for k in node] == [full_stats[k] for k in node]


def test_visit_range_arguments(cuda_ok):
    t = _particles("cuda")
    n = len(t["x"])
    with ct.TreePmCoordinator(_config(ct._abi.FP64)) as s:
        with pytest.raises(ct.StateError):
            s.visit_order(0, 64)
        with pytest.raises(ct.StateError):
            s.walk_cost(0, 64)
        for bad in ((32, 128), (0, 100), (-64, 64), (128, 64), (0, n + 64)):
            with pytest.raises(ct.InvalidArgument):
                s.solve_active_set(t["x"], t["y"], t["z"], t["m"], visit_range=bad)
        # an empty slice at the end and a slice ending at the target count are valid
        r = s.solve_active_set(t["x"], t["y"], t["z"], t["m"], visit_range=(n, n))
        assert r["ax"].numel() == 0
        r = s.solve_active_set(t["x"], t["y"], t["z"], t["m"], visit_range=(n - 64 * 3, n))
        assert r["ax"].numel() == 64 * 3 and bool(torch.isfinite(r["ax"]).all())
        with pytest.raises(ct.InvalidArgument):
            s.visit_order(0, n + 1)
        with pytest.raises(ct.InvalidArgument):
            s.walk_cost(16, 64)


def test_active_set_slices(cuda_ok):
    """Slices of an active set's visit order (active slots sorted by tree position)."""
    t = _particles("cuda")
    n = len(t["x"])
    active = torch.arange(0, n, 3, device="cuda")
    with ct.TreePmCoordinator(_config(ct._abi.FP64)) as s:
        full = s.solve_active_set(t["x"], t["y"], t["z"], t["m"], active=active)
        na = len(active)
        order = s.visit_order(0, na, device="cuda")
        assert torch.equal(torch.sort(order).values, torch.arange(na, device="cuda"))
        got = torch.full((na,), float("nan"), dtype=torch.float64, device="cuda")
        bounds = sharded.even_bounds(na, 4)
        for q in range(4):
            b, e = bounds[q], bounds[q + 1]
            r = s.solve_active_set_with_pm_cadence(t["x"], t["y"], t["z"], t["m"], False, active=active,
                                                   visit_range=(b, e))
            got[order[b:e]] = r["ax"]
    assert float((got - full["ax"]).abs().max()) <= 1e-12 * float(full["ax"].abs().max())


def _kdk(solver, t, acc, factors, steps, shard=None):
    d, k1, k2, g1, g2 = factors
    for _ in range(steps):
        solver.kick(t["vx"], t["vy"], t["vz"], acc[0], acc[1], acc[2], k1, g1)
        solver.drift(t["x"], t["y"], t["z"], t["vx"], t["vy"], t["vz"], d)
        if shard is None:
            r = solver.solve_active_set(t["x"], t["y"], t["z"], t["m"])
            acc = (r["ax"], r["ay"], r["az"])
        else:
            acc = shard.accelerations(t["x"], t["y"], t["z"], t["m"])
        solver.kick(t["vx"], t["vy"], t["vz"], acc[0], acc[1], acc[2], k2, g2)
    return acc


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, os.path.join(ROOT, "chui-dev_b200"))
    import torch.distributed as dist

    import chui_treepm as ctr
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        torch.cuda.set_device(0)
        t = _particles("cuda")
        with ctr.TreePmCoordinator(_config(ctr._abi.FP64, 0)) as s:
            shard = ctr.ShardedTreePm(s)
            acc = shard.accelerations(t["x"], t["y"], t["z"], t["m"])
            _kdk(s, t, acc, ctr.kdk_factors_static(0.02), 3, shard)
            out[rank] = {k: t[k].cpu().numpy() for k in ("x", "y", "z", "vx")} | {"bounds": shard.bounds}
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_processes_step_one_simulation(cuda_ok):
    import torch.multiprocessing as mp
    t = _particles("cuda")
    with ct.TreePmCoordinator(_config(ct._abi.FP64, 0)) as s:
        r = s.solve_active_set(t["x"], t["y"], t["z"], t["m"])
        _kdk(s, t, (r["ax"], r["ay"], r["az"]), ct.kdk_factors_static(0.02), 3)
    want = {k: t[k].cpu().numpy() for k in ("x", "y", "z", "vx")}
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as manager:
        out = manager.dict()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=300)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        out = dict(out)
    # both ranks hold the same state, bit for bit
    for k in ("x", "y", "z", "vx"):
        assert np.array_equal(out[0][k], out[1][k]), k
    # and it is the single-process state (the PM deposit's FP64 atomics may round differently)
    for k in ("x", "y", "z"):
        d = np.abs(out[0][k] - want[k])
        d = np.minimum(d, BOX - d)
        assert d.max() <= 1e-10 * BOX, (k, d.max())
    assert np.abs(out[0]["vx"] - want["vx"]).max() <= 1e-9 * np.abs(want["vx"]).max()
    assert out[0]["bounds"][0] == 0 and out[0]["bounds"][-1] == N_SIDE ** 3
