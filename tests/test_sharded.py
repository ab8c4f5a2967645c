"""Target-sharded TreePM on CPU (chui_treepm.sharded): slice boundaries, cost
balancing, and the accelerations' all-gather over gloo ranks (world sizes 2
and 3) with a stand-in solver whose visit order and forces are known. The
library's own visit-range solve is checked on the GPU
(tests/test_gpu_sharded.py)."""
import os
import socket
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "chui-dev_b200"))

from chui_treepm import sharded  # noqa: E402


def test_even_bounds_are_aligned_and_cover():
    for n, world in ((1000, 3), (64, 4), (10, 2), (1 << 20, 8), (0, 2)):
        b = sharded.even_bounds(n, world)
        assert b[0] == 0 and b[-1] == n and len(b) == world + 1
        assert all(b[i] <= b[i + 1] for i in range(world))
        assert all(v % 64 == 0 or v == n for v in b)


def test_balanced_bounds_equalise_a_skewed_cost():
    # cost density over visit positions: a dense clump in the first quarter
    n, world = 1 << 16, 4
    dens = np.ones(n)
    dens[: n // 4] = 20.0
    cum = np.concatenate([[0.0], np.cumsum(dens)])
    bounds = sharded.even_bounds(n, world)
    for _ in range(6):
        costs = [cum[bounds[q + 1]] - cum[bounds[q]] for q in range(world)]
        bounds = sharded.balanced_bounds(bounds, costs)
        assert bounds[0] == 0 and bounds[-1] == n
        assert all(v % 64 == 0 or v == n for v in bounds)
        assert all(bounds[i] <= bounds[i + 1] for i in range(world))
    costs = [cum[bounds[q + 1]] - cum[bounds[q]] for q in range(world)]
    assert max(costs) / min(costs) < 1.05, costs


def test_balanced_bounds_fall_back_to_even():
    b = sharded.even_bounds(4096, 4)
    assert sharded.balanced_bounds(b, [0.0, 0.0, 0.0, 0.0]) == b
    assert sharded.balanced_bounds(b, [1.0, float("nan"), 1.0, 1.0]) == b
    with pytest.raises(ValueError):
        sharded.balanced_bounds(b, [1.0, 1.0])


class FakeSolver:
    """Visit order = positions sorted by x; 'force' = a known function of the
    position; walk cost = a known per-target cost summed over the slice."""

    def __init__(self, perturb=False):
        self.last_stats = {}
        self.perturb = perturb

    def solve_active_set_with_pm_cadence(self, x, y, z, m, refresh, uniform_mass=None, visit_range=None,
                                         stream=None):
        order = torch.argsort(x, stable=True)
        if self.perturb:
            order = order.flip(0)
        self._order = order
        b, e = visit_range
        sl = order[b:e]
        cost = 1.0 + 9.0 * (x[sl] < 0.2).to(torch.float64)
        self.last_stats = {"walk_ms": float(cost.sum())}
        return {"ax": torch.sin(x[sl]), "ay": torch.cos(y[sl]), "az": x[sl] * z[sl]}

    def visit_order(self, b, e, device=None):
        return self._order[b:e].clone()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n, out, perturb_rank):
    sys.path.insert(0, os.path.join(ROOT, "chui-dev_b200"))
    from chui_treepm import sharded as sh
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        g = torch.Generator().manual_seed(7)
        x, y, z = (torch.rand(n, generator=g, dtype=torch.float64) for _ in range(3))
        m = torch.full((n,), 1.0 / n, dtype=torch.float64)
        s = sh.ShardedTreePm(FakeSolver(perturb=(rank == perturb_rank)))
        res = {}
        try:
            for step in range(3):
                ax, ay, az = s.accelerations(x, y, z, m)
                ok = (torch.equal(ax, torch.sin(x)) and torch.equal(ay, torch.cos(y)) and torch.equal(az, x * z))
                res[f"ok{step}"] = ok
            res["bounds"] = list(s.bounds)
            res["counts"] = list(s.last_counts)
            res["walk"] = list(s.last_walk_ms)
        except RuntimeError as exc:
            res["error"] = str(exc)
        out[rank] = res
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _run(world, n, perturb_rank=-1):
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as manager:
        out = manager.dict()
        procs = [ctx.Process(target=_worker, args=(r, world, port, n, out, perturb_rank)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=180)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        return dict(out)


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_accelerations_assemble_on_every_rank(world):
    n = 5000
    out = _run(world, n)
    for r in range(world):
        assert all(out[r][f"ok{k}"] for k in range(3)), out[r]
        # every rank computes the same boundaries
        assert out[r]["bounds"] == out[0]["bounds"]
    # balancing on slice totals moves toward equal cost step by step
    walk = out[0]["walk"]
    assert max(walk) / min(walk) < 3.0, walk
    assert sum(out[0]["counts"]) == n


def test_diverged_visit_order_is_detected_on_every_rank():
    out = _run(2, 3000, perturb_rank=1)
    for r in range(2):
        assert "visit order" in out[r].get("error", ""), out[r]


def test_single_rank_without_process_group():
    n = 1000
    x, y, z = (torch.linspace(0.0, 1.0, n, dtype=torch.float64) for _ in range(3))
    s = sharded.ShardedTreePm(FakeSolver(), group=False)
    ax, ay, az = s.accelerations(x, y, z, torch.ones(n, dtype=torch.float64))
    assert s.world == 1 and s.bounds == [0, n]
    assert torch.equal(ax, torch.sin(x)) and torch.equal(az, x * z)


def test_profile_bounds_cut_equal_cost():
    rng = np.random.default_rng(3)
    n, world = 100_000, 8
    cost = rng.gamma(0.3, 1.0, (n + 31) // 32)
    b = sharded.profile_bounds(cost, n, world)
    assert b[0] == 0 and b[-1] == n and all(v % 64 == 0 or v == n for v in b)
    cum = np.concatenate([[0.0], np.cumsum(cost)])
    part = [cum[b[q + 1] // 32 if b[q + 1] < n else len(cost)] - cum[b[q] // 32] for q in range(world)]
    # within two chunks' cost of the ideal share
    assert max(abs(p - cum[-1] / world) for p in part) <= 2.0 * cost.max() + 1e-9
    assert sharded.profile_bounds(np.zeros_like(cost), n, world) == sharded.even_bounds(n, world)
    with pytest.raises(ValueError):
        sharded.profile_bounds(cost[:-1], n, world)


class ProfiledSolver(FakeSolver):
    """FakeSolver that also reports a per-32-position cost profile."""

    def solve_active_set_with_pm_cadence(self, x, y, z, m, refresh, uniform_mass=None, visit_range=None,
                                         stream=None):
        r = super().solve_active_set_with_pm_cadence(x, y, z, m, refresh, uniform_mass, visit_range, stream)
        b, e = visit_range
        cost = 1.0 + 9.0 * (x[self._order[b:e]] < 0.2).to(torch.float64)
        pad = (-len(cost)) % 32
        self._profile = torch.cat([cost, torch.zeros(pad, dtype=torch.float64)]).view(-1, 32).sum(1)
        return r

    def walk_cost(self, b, e, device=None):
        return self._profile.to(torch.float32)


def _worker_profiled(rank, world, port, n, out):
    sys.path.insert(0, os.path.join(ROOT, "chui-dev_b200"))
    from chui_treepm import sharded as sh
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        g = torch.Generator().manual_seed(11)
        x, y, z = (torch.rand(n, generator=g, dtype=torch.float64) for _ in range(3))
        s = sh.ShardedTreePm(ProfiledSolver())
        ok = True
        for _ in range(2):
            ax, ay, az = s.accelerations(x, y, z, torch.ones(n, dtype=torch.float64))
            ok = ok and torch.equal(ax, torch.sin(x)) and torch.equal(az, x * z)
        out[rank] = {"ok": ok, "walk": list(s.last_walk_ms), "bounds": list(s.bounds)}
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_profile_balances_in_one_step():
    # large enough that the 64-position alignment is a small part of a slice
    world, n = 3, 60000
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as manager:
        out = manager.dict()
        procs = [ctx.Process(target=_worker_profiled, args=(r, world, port, n, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=180)
        assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
        out = dict(out)
    for r in range(world):
        assert out[r]["ok"] and out[r]["bounds"] == out[0]["bounds"]
    walk = out[0]["walk"]  # the second force used the profile of the first
    assert max(walk) / min(walk) < 1.1, walk
