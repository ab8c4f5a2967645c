"""One TreePM simulation across the ranks of a process group (one process per
GPU): sources replicated, targets sharded.

Every rank holds the whole particle state (FP64 positions and velocities and
the masses: 56 bytes per particle, 0.94 GB at 256^3 and 7.5 GB at 512^3 of a
B200's 180 GB), builds the same tree and PM field from it, and walks one slice
of the common visit order (`chui_treepm_solve_visit_range`). One all-gather per
force assembles the slices' accelerations (24 bytes per particle) on every
rank, which then kicks and drifts every particle identically, so the state
stays the same on all ranks without further exchange. The residual walk, about
90 % of a force, divides across the ranks; the PM refresh and the tree build
are repeated on each.

The reference splits the same computation differently: MPI ranks own their
particles, the PM mesh is slab-decomposed and each rank imports a locally
essential tree from the others (tree_pm_coupling.cpp:2282-3518 with the
PmSlabLayout of pm_solver.hpp). Inside one NVSwitch node, with every rank
able to hold every particle, replicating the sources costs one all-gather of
the accelerations per force and no ghost or slab exchange.

Slices are balanced on the walk's own device time: the walk records the SM
cycles it spent on every block of 32 visit positions (`chui_treepm_walk_cost`),
the ranks exchange their slices' profiles, and the next boundaries cut the
cumulative cost into equal parts (rounded to the 64-target blocks the walk
groups targets in). Visit positions map to the same regions of the box from
one step to the next (tree order), so the profile carries over. Where no profile is recorded (a solver
without one, diagnostics on, several masses) the slices are balanced on their
total walk times instead, each spread evenly over its slice.

The visit order itself must be the same on every rank (same positions, same
tree); each force checks it with a hash compared across ranks and raises
`RuntimeError` when the ranks disagree.
"""
from __future__ import annotations

import math

ALIGN = 64  # visit-range ends: multiples of the walk's residual blocks


def even_bounds(n: int, world: int, align: int = ALIGN) -> list[int]:
    """Boundaries b_0 = 0 <= ... <= b_world = n of equal slices, inner ones
    rounded to multiples of `align` (a rounded value beyond n becomes n)."""
    out = [0]
    for k in range(1, world):
        b = int(round(n * k / world / align)) * align
        out.append(min(max(b, out[-1]), n))
    out.append(n)
    return out


def balanced_bounds(bounds: list[int], costs: list[float], align: int = ALIGN) -> list[int]:
    """New boundaries that cut the cumulative cost into len(costs) equal
    parts. Slice q's cost costs[q] is spread evenly over its positions
    [bounds[q], bounds[q+1]); empty slices carry no cost. Non-finite or
    non-positive totals give even slices."""
    world = len(costs)
    n = bounds[-1]
    if len(bounds) != world + 1:
        raise ValueError("one cost per slice")
    total = sum(costs)
    if not (math.isfinite(total) and total > 0.0) or any(not math.isfinite(c) or c < 0.0 for c in costs):
        return even_bounds(n, world, align)
    out = [0]
    q = 0
    below = 0.0  # cost of the slices before q
    for k in range(1, world):
        target = total * k / world
        while q < world - 1 and below + costs[q] < target:
            below += costs[q]
            q += 1
        width = bounds[q + 1] - bounds[q]
        frac = (target - below) / costs[q] if costs[q] > 0.0 else 0.0
        pos = bounds[q] + min(max(frac, 0.0), 1.0) * width
        b = int(round(pos / align)) * align
        out.append(min(max(b, out[-1]), n))
    out.append(n)
    return out


def profile_bounds(chunk_cost, n: int, world: int, align: int = ALIGN) -> list[int]:
    """Boundaries at equal fractions of a measured cost profile: chunk_cost[k]
    is the cost of visit positions [32k, 32k + 32) (the whole range, in
    order). Each boundary is the aligned position nearest the point where the
    cumulative cost crosses k / world of the total. A profile without
    positive finite cost gives even slices."""
    import numpy as np

    cost = np.asarray(chunk_cost, dtype=np.float64)
    if cost.size != (n + 31) // 32:
        raise ValueError("one cost per 32 visit positions")
    total = float(cost.sum()) if cost.size else 0.0
    if not (np.isfinite(total) and total > 0.0) or (cost < 0.0).any():
        return even_bounds(n, world, align)
    cum = np.cumsum(cost)
    out = [0]
    for k in range(1, world):
        target = total * k / world
        c = int(np.searchsorted(cum, target))  # first chunk whose end reaches the target
        before = float(cum[c - 1]) if c > 0 else 0.0
        frac = (target - before) / cost[c] if cost[c] > 0.0 else 0.0
        pos = 32.0 * (c + min(max(frac, 0.0), 1.0))
        b = int(round(pos / align)) * align
        out.append(min(max(b, out[-1]), n))
    out.append(n)
    return out


def hash_weights(torch, n: int, device):
    """Per-position weights of `order_hash`."""
    idx = torch.arange(n, device=device, dtype=torch.int64)
    return (idx * 2654435761 + 97) & 0x7FFFFFFF


def order_hash(torch, order, weights=None) -> int:
    """A 64-bit fingerprint of a visit order (weighted sum, wrapping)."""
    w = hash_weights(torch, order.numel(), order.device) if weights is None else weights
    return int((order * w).sum().item())


class ShardedTreePm:
    """Target-sharded forces for one simulation replicated on every rank.

    solver: a `TreePmCoordinator` on this rank's GPU (or any object with its
    `solve_active_set_with_pm_cadence(..., visit_range=)`, `visit_order` and
    `last_stats`). group: a torch.distributed process group, None for the
    default one, or False for a single rank without torch.distributed.
    """

    def __init__(self, solver, group=None, balance: bool = True, verify: bool = True):
        import torch
        import torch.distributed as dist

        self.torch = torch
        self.solver = solver
        self.balance = balance
        self.verify = verify
        if group is False or not dist.is_available() or not dist.is_initialized():
            self.dist, self.group, self.rank, self.world = None, None, 0, 1
        else:
            self.dist = dist
            self.group = group
            self.rank = dist.get_rank(group)
            self.world = dist.get_world_size(group)
        self.bounds: list[int] | None = None
        self._weights = None
        self.last_walk_ms: list[float] = []
        self.last_counts: list[int] = []

    # -- communication ------------------------------------------------------
    def _comm_device(self, like):
        """NCCL moves CUDA tensors; other backends (gloo) move host tensors."""
        if self.dist is None:
            return like.device
        backend = self.dist.get_backend(self.group)
        return like.device if backend == "nccl" else self.torch.device("cpu")

    def _all_gather(self, t):
        """all-gather of equal-shaped tensors -> (world, *t.shape) on t's device."""
        torch = self.torch
        if self.dist is None:
            return t.unsqueeze(0)
        dev = self._comm_device(t)
        src = t.to(dev).contiguous()
        if dev.type == "cuda":
            out = torch.empty((self.world,) + tuple(src.shape), dtype=src.dtype, device=dev)
            self.dist.all_gather_into_tensor(out, src, group=self.group)
        else:
            parts = [torch.empty_like(src) for _ in range(self.world)]
            self.dist.all_gather(parts, src, group=self.group)
            out = torch.stack(parts)
        return out.to(t.device)

    # -- the force ------------------------------------------------------------
    def slice_of(self, rank: int) -> tuple[int, int]:
        return self.bounds[rank], self.bounds[rank + 1]

    def accelerations(self, x, y, z, mass, uniform_mass=None, refresh_long_range_field: bool = True,
                      stream=None):
        """Total accelerations of every particle (particle order), identical on
        every rank: this rank's slice is solved here, the rest arrive by one
        all-gather. x, y, z, mass are this rank's full copies (torch tensors)."""
        torch = self.torch
        n = len(x)
        if self.bounds is None or self.bounds[-1] != n or len(self.bounds) != self.world + 1:
            self.bounds = even_bounds(n, self.world)
        b, e = self.slice_of(self.rank)
        r = self.solver.solve_active_set_with_pm_cadence(x, y, z, mass, refresh_long_range_field,
                                                         uniform_mass=uniform_mass, visit_range=(b, e),
                                                         stream=stream)
        walk_ms = float(self.solver.last_stats.get("walk_ms", 0.0))
        order = self.solver.visit_order(0, n, device=x.device if x.is_cuda else None)
        if not torch.is_tensor(order):
            order = torch.from_numpy(order.astype("int64"))
        order = order.to(x.device)

        # the slices' accelerations, padded to the longest slice
        counts = [self.bounds[q + 1] - self.bounds[q] for q in range(self.world)]
        width = max(counts) if counts else 0
        local = torch.empty((3, width), dtype=torch.float64, device=x.device)  # the padding is never read
        local[0, : e - b] = r["ax"]
        local[1, : e - b] = r["ay"]
        local[2, : e - b] = r["az"]
        gathered = self._all_gather(local)  # (world, 3, width)
        vis = torch.cat([gathered[q, :, : counts[q]] for q in range(self.world)], dim=1)
        acc = torch.empty((3, n), dtype=torch.float64, device=x.device)
        acc.index_copy_(1, order, vis)

        # per rank: walk time, visit-order fingerprint (two exact 32-bit
        # halves) and, when the solver reports it, the walk's cycles per 32
        # visit positions of its slice; one small all-gather
        chunks = [(c + 31) // 32 for c in counts]
        profile = None
        if hasattr(self.solver, "walk_cost"):
            profile = self.solver.walk_cost(b, e, device=x.device if x.is_cuda else None)
            if not torch.is_tensor(profile):
                profile = torch.from_numpy(profile)
        info = torch.zeros(3 + max(chunks), dtype=torch.float64, device=x.device)
        info[0] = walk_ms
        h = 0
        if self.verify:
            if self._weights is None or self._weights.numel() != n or self._weights.device != order.device:
                self._weights = hash_weights(torch, n, order.device)
            h = order_hash(torch, order, self._weights)
        info[1] = float(h & 0xFFFFFFFF)
        info[2] = float((h >> 32) & 0xFFFFFFFF)
        if profile is not None:
            info[3 : 3 + profile.numel()] = profile.to(device=x.device, dtype=torch.float64)
        infos = self._all_gather(info).cpu()
        self.last_walk_ms = [float(v) for v in infos[:, 0]]
        self.last_counts = counts
        if self.verify and not (torch.equal(infos[:, 1], infos[:1, 1].expand(self.world)) and
                                torch.equal(infos[:, 2], infos[:1, 2].expand(self.world))):
            raise RuntimeError("ranks disagree on the visit order: the replicated particle state has diverged")
        if self.balance and self.world > 1:
            full = None
            if profile is not None:
                full = torch.cat([infos[q, 3 : 3 + chunks[q]] for q in range(self.world)]).numpy()
            if full is not None and full.sum() > 0.0:
                self.bounds = profile_bounds(full, n, self.world)
            else:  # no profile recorded (diagnostics on, several masses, ...): slice totals
                self.bounds = balanced_bounds(self.bounds, self.last_walk_ms)
        return acc[0], acc[1], acc[2]
