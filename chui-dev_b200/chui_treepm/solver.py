"""Python mirror of the reference's TreePM gravity-solver interface over the
C-ABI (include/chui_treepm.h).

`TreePmCoordinator` follows cosmosim::gravity::TreePmCoordinator
(include/cosmosim/gravity/tree_pm_coupling.hpp:527-814 in the reference):
construct with the mesh shape and options, then `solve_active_set` /
`solve_active_set_with_pm_cadence` with source positions, masses and an
accumulator. Errors carry the reference's exception types: invalid input
raises ValueError (std::invalid_argument), index/depth/stack overflow raises
IndexError / OverflowError (std::out_of_range / std::overflow_error), reuse of
a missing PM field raises RuntimeError (std::runtime_error).

Arrays may be numpy arrays (host memory: the library stages them) or CUDA
torch tensors of the context's device (device memory: used in place, the
zero-copy path).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, fields

import numpy as np

from . import _abi


class TreePmError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


class InvalidArgument(TreePmError, ValueError):
    pass


class OutOfRange(TreePmError, IndexError):
    pass


class StateError(TreePmError):
    pass


class DeviceError(TreePmError):
    pass


class AllocationError(TreePmError, MemoryError):
    pass


class NotSupported(TreePmError, NotImplementedError):
    pass


_ERRORS = {
    _abi.EINVAL: InvalidArgument,
    _abi.ERANGE: OutOfRange,
    _abi.ESTATE: StateError,
    _abi.EDEVICE: DeviceError,
    _abi.ENOMEM: AllocationError,
    _abi.ENOTSUP: NotSupported,
}


@dataclass
class TreePmConfig:
    """The `.param.txt` [numerics] treepm_* knobs (see chui_treepm.config)."""
    pm_grid_nx: int = 16
    pm_grid_ny: int = 16
    pm_grid_nz: int = 16
    box_x: float = 1.0
    box_y: float = 1.0
    box_z: float = 1.0
    asmth_cells: float = 1.25
    rcut_cells: float = 6.25
    opening_theta: float = 0.7
    opening_criterion: int = _abi.OPEN_COM_DISTANCE
    multipole_order: int = 2
    max_leaf_size: int = 16
    assignment_scheme: int = _abi.CIC
    window_deconvolution: int = 0
    gravitational_constant: float = 1.0
    softening: float = 0.0
    acceptance_policy: int = _abi.POLICY_STRICT
    precision: int = _abi.MIXED
    device: int = 0
    diagnostics: int = 0
    adaptive_error_estimator: int = _abi.ESTIMATOR_RESIDUAL_DERIVATIVE
    cutoff_node_policy: int = _abi.CUTOFF_CONTAIN_NODE
    adaptive_maximum_opening_angle: float = 0.25
    relative_force_tolerance: float = 0.005
    relative_force_acceleration_floor: float = 1.0e-30
    group_walk_enabled: int = 0
    gaussian_pair_lookup: int = 0
    boundary_condition: int = _abi.BOUNDARY_PERIODIC
    short_range_only: int = 0

    def to_c(self) -> _abi.Config:
        c = _abi.Config()
        for f in fields(self):
            setattr(c, f.name, getattr(self, f.name))
        return c

    @property
    def mesh_spacing(self) -> float:
        return ((self.box_x / self.pm_grid_nx) * (self.box_y / self.pm_grid_ny) *
                (self.box_z / self.pm_grid_nz)) ** (1.0 / 3.0)


def _is_torch(a) -> bool:
    return hasattr(a, "data_ptr") and hasattr(a, "is_cuda")


class _Arrays:
    """Resolves numpy / torch inputs to raw pointers for one call."""

    def __init__(self, sample):
        self.device = _is_torch(sample) and sample.is_cuda
        self.keep = []

    def ptr(self, a, dtype):
        if a is None:
            return None
        if self.device:
            import torch
            if not (_is_torch(a) and a.is_cuda):
                raise InvalidArgument(_abi.EINVAL, "mixed host and device arrays in one call")
            if dtype == np.uint32:
                # 32-bit index lanes travel as int32 bit patterns (0xFFFFFFFF == -1)
                if a.dtype != torch.int32:
                    a = a.to(torch.int64)
                    a = torch.where(a >= 2 ** 31, a - 2 ** 32, a).to(torch.int32)
            elif dtype == np.float64:
                if a.dtype != torch.float64:
                    a = a.to(torch.float64)
            elif a.dtype != torch.int64:
                a = a.to(torch.int64)
            a = a.contiguous()
            self.keep.append(a)
            return a.data_ptr()
        arr = np.ascontiguousarray(a, dtype=dtype)
        self.keep.append(arr)
        return arr.ctypes.data

    def out_into(self, a, n):
        """A caller-provided FP64 output of n entries (same memory kind as the inputs)."""
        if self.device:
            if not (_is_torch(a) and a.is_cuda and a.dtype.itemsize == 8 and a.is_contiguous() and a.numel() == n):
                raise InvalidArgument(_abi.EINVAL, "output tensors must be contiguous FP64 CUDA tensors of the target count")
            self.keep.append(a)
            return a, a.data_ptr()
        if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous and a.size == n):
            raise InvalidArgument(_abi.EINVAL, "output arrays must be contiguous float64 arrays of the target count")
        self.keep.append(a)
        return a, a.ctypes.data

    def out(self, n, like=None, dtype=np.float64):
        if self.device:
            import torch
            t = torch.empty(n, dtype=torch.float64 if dtype == np.float64 else torch.int64, device=like.device)
            self.keep.append(t)
            return t, t.data_ptr()
        arr = np.empty(n, dtype=dtype)
        self.keep.append(arr)
        return arr, arr.ctypes.data


class TreePmCoordinator:
    """B200 TreePM solver instance (owns PM mesh, FFT plans, tree, scratch)."""

    def __init__(self, config: TreePmConfig):
        self._lib = _abi.load()
        self.config = config
        h = C.c_void_p()
        rc = self._lib.chui_treepm_create(C.byref(config.to_c()), C.byref(h))
        if rc != 0:
            msg = self._lib.chui_treepm_last_error(None).decode()
            raise _ERRORS.get(rc, TreePmError)(rc, msg or f"chui_treepm_create failed ({rc})")
        self._h = h
        self.last_stats: dict = {}

    def close(self):
        if getattr(self, "_h", None):
            self._lib.chui_treepm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int):
        if rc != 0:
            msg = self._lib.chui_treepm_last_error(self._h).decode()
            raise _ERRORS.get(rc, TreePmError)(rc, msg or f"error {rc}")

    def set_config(self, config: TreePmConfig):
        self._check(self._lib.chui_treepm_set_config(self._h, C.byref(config.to_c())))
        self.config = config

    # -- solve ----------------------------------------------------------------
    def solve_active_set_with_pm_cadence(self, x, y, z, mass, refresh_long_range_field: bool, active=None,
                                         targets=None, uniform_mass: float | None = None,
                                         long_range: bool = False, short_range: bool = False,
                                         nearest_pair: bool = False, previous_acceleration=None,
                                         out=None, stream=None, visit_range=None, softening=None,
                                         target_softening=None) -> dict:
        """TreePmCoordinator::solveActiveSetWithPmCadence. Returns a dict with
        ax, ay, az (active-slot order) and the requested optional lanes.
        previous_acceleration: per active slot |a_previous| for the relative
        criteria (NaN entries: no history for that target), or None.
        out: optional (ax, ay, az) arrays to write into (the accumulator's
        accel spans; pinned host arrays make the device-to-host copy a DMA).
        visit_range: (begin, end) walks only the targets at those visit
        positions (chui_treepm_solve_visit_range); ax.. and pm_a.. then hold
        end - begin entries in visit order (visit_order(begin, end) gives
        their slots).
        softening / target_softening: resolved per-source and per-active-slot
        Plummer epsilons (chui_treepm.softening resolves a TreeSofteningView
        into them), or None for config.softening."""
        arr = _Arrays(x)
        n = len(x)
        src = _abi.Sources()
        src.count = n
        src.x, src.y, src.z = arr.ptr(x, np.float64), arr.ptr(y, np.float64), arr.ptr(z, np.float64)
        if mass is None:
            if uniform_mass is None:
                raise InvalidArgument(_abi.EINVAL, "mass or uniform_mass is required")
            src.mass = None
            src.uniform_mass = float(uniform_mass)
        else:
            src.mass = arr.ptr(mass, np.float64)
            src.uniform_mass = 0.0
        acc = _abi.Accumulator()
        if targets is not None:
            tx, ty, tz = targets
            nt = len(tx)
            acc.target_x, acc.target_y, acc.target_z = (arr.ptr(tx, np.float64), arr.ptr(ty, np.float64),
                                                        arr.ptr(tz, np.float64))
            if active is None:
                active = np.full(nt, 0xFFFFFFFF, dtype=np.uint32)
                if arr.device:
                    import torch
                    active = torch.full((nt,), 0xFFFFFFFF, dtype=torch.int64, device=x.device)
        else:
            nt = n if active is None else len(active)
        acc.active_count = nt
        acc.active_index = arr.ptr(active, np.uint32) if active is not None else None
        if softening is not None:
            if len(softening) != n:
                raise InvalidArgument(_abi.EINVAL, "TreePM source softening sidecar size must match source particle count")
            src.softening = arr.ptr(softening, np.float64)
        if target_softening is not None:
            if len(target_softening) != nt:
                raise InvalidArgument(_abi.EINVAL, "TreePM target softening sidecar size must match active-set size")
            acc.target_softening = arr.ptr(target_softening, np.float64)
        if previous_acceleration is not None:
            if len(previous_acceleration) != nt:
                raise InvalidArgument(_abi.EINVAL, "TreePM force accumulator spans must have matching active-set extent")
            acc.previous_acceleration_magnitude = arr.ptr(previous_acceleration, np.float64)
        nout = nt
        if visit_range is not None:
            begin, end = (int(v) for v in visit_range)
            nout = max(end - begin, 0)
        given = out
        out = {}
        if given is not None:
            if len(given) != 3:
                raise InvalidArgument(_abi.EINVAL, "out takes the three acceleration arrays")
            out["ax"], acc.accel_x = arr.out_into(given[0], nout)
            out["ay"], acc.accel_y = arr.out_into(given[1], nout)
            out["az"], acc.accel_z = arr.out_into(given[2], nout)
        else:
            out["ax"], acc.accel_x = arr.out(nout, x)
            out["ay"], acc.accel_y = arr.out(nout, x)
            out["az"], acc.accel_z = arr.out(nout, x)
        if long_range:
            out["pm_ax"], acc.long_range_x = arr.out(nout, x)
            out["pm_ay"], acc.long_range_y = arr.out(nout, x)
            out["pm_az"], acc.long_range_z = arr.out(nout, x)
        if short_range:
            for k, attr in (("tree_ax", "short_range_x"), ("tree_ay", "short_range_y"),
                            ("tree_az", "short_range_z")):
                a, p = arr.out(n, x)
                a[:] = 0.0
                out[k] = a
                setattr(acc, attr, p)
        if nearest_pair:
            a, p = arr.out(n, x)
            a[:] = float("inf")
            out["nearest_r2"] = a
            acc.nearest_pair_r2 = p
        st = _abi.Stats()
        mem = _abi.DEVICE if arr.device else _abi.HOST
        strm = C.c_void_p(stream) if stream else None
        refresh = 1 if refresh_long_range_field else 0
        if visit_range is None:
            rc = self._lib.chui_treepm_solve(self._h, C.byref(src), C.byref(acc), refresh, mem, strm, C.byref(st))
        else:
            rc = self._lib.chui_treepm_solve_visit_range(self._h, C.byref(src), C.byref(acc), refresh, mem, strm,
                                                         C.byref(st), begin, end)
        self._check(rc)
        self.last_stats = st.as_dict()
        out["stats"] = self.last_stats
        return out

    def solve_active_set(self, x, y, z, mass, **kw) -> dict:
        """TreePmCoordinator::solveActiveSet: the cadence variant with refresh."""
        return self.solve_active_set_with_pm_cadence(x, y, z, mass, True, **kw)

    def visit_order(self, begin: int, end: int, device=None):
        """Slots (particle rows for a full solve) at visit positions
        [begin, end) of the last solve: a uint32 numpy array, or an int64 CUDA
        tensor on `device`."""
        n = max(int(end) - int(begin), 0)
        if device is None:
            out = np.empty(n, dtype=np.uint32)
            self._check(self._lib.chui_treepm_visit_order(self._h, int(begin), int(end),
                                                          C.c_void_p(out.ctypes.data), _abi.HOST, None))
            return out
        import torch
        out = torch.empty(n, dtype=torch.int32, device=device)
        self._check(self._lib.chui_treepm_visit_order(self._h, int(begin), int(end), C.c_void_p(out.data_ptr()),
                                                      _abi.DEVICE, None))
        # uint32 bit patterns; rows stay below 2^32 - 1
        return out.to(torch.int64) & 0xFFFFFFFF

    def walk_cost(self, begin: int, end: int, device=None):
        """SM cycles the last solve's walk spent per 32 visit positions from
        `begin` (a multiple of 32) to `end`: float32 numpy array, or a CUDA
        tensor on `device`."""
        n = (max(int(end) - int(begin), 0) + 31) // 32
        if device is None:
            out = np.zeros(n, dtype=np.float32)
            self._check(self._lib.chui_treepm_walk_cost(self._h, int(begin), int(end),
                                                        C.c_void_p(out.ctypes.data), _abi.HOST, None))
            return out
        import torch
        out = torch.zeros(n, dtype=torch.float32, device=device)
        self._check(self._lib.chui_treepm_walk_cost(self._h, int(begin), int(end), C.c_void_p(out.data_ptr()),
                                                    _abi.DEVICE, None))
        return out

    # -- PM pieces ------------------------------------------------------------
    def assign_density(self, x, y, z, mass, uniform_mass: float = 0.0):
        arr = _Arrays(x)
        src = _abi.Sources()
        src.count = len(x)
        src.x, src.y, src.z = arr.ptr(x, np.float64), arr.ptr(y, np.float64), arr.ptr(z, np.float64)
        src.mass = arr.ptr(mass, np.float64) if mass is not None else None
        src.uniform_mass = uniform_mass
        c = self.config
        rho, p = arr.out(c.pm_grid_nx * c.pm_grid_ny * c.pm_grid_nz, x)
        self._check(self._lib.chui_pm_assign_density(self._h, C.byref(src), C.c_void_p(p),
                                                     _abi.DEVICE if arr.device else _abi.HOST, None))
        return rho

    def cells(self, x, y, z):
        arr = _Arrays(x)
        src = _abi.Sources()
        src.count = len(x)
        src.x, src.y, src.z = arr.ptr(x, np.float64), arr.ptr(y, np.float64), arr.ptr(z, np.float64)
        out, p = arr.out(3 * len(x), x, dtype=np.int64)
        self._check(self._lib.chui_pm_cells(self._h, C.byref(src), C.c_void_p(p),
                                            _abi.DEVICE if arr.device else _abi.HOST, None))
        return out.reshape(-1, 3)

    # -- parity dumps ---------------------------------------------------------
    def dump_tree(self, n: int) -> dict:
        nn = C.c_int64()
        self._check(self._lib.chui_treepm_tree_node_count(self._h, C.byref(nn)))
        nn = nn.value
        d = _abi.TreeDump()
        r = {}
        for k in ("center_x", "center_y", "center_z", "half_size", "mass", "com_x", "com_y", "com_z",
                  "quad_xx", "quad_xy", "quad_xz", "quad_yy", "quad_yz", "quad_zz", "second_moment_trace"):
            r[k] = np.zeros(nn)
            setattr(d, k, r[k].ctypes.data)
        for k, cnt in (("child_count", nn), ("child_index", 8 * nn), ("particle_begin", nn),
                       ("particle_count", nn)):
            r[k] = np.zeros(cnt, dtype=np.uint32)
            setattr(d, k, r[k].ctypes.data)
        self._check(self._lib.chui_treepm_dump_tree(self._h, C.byref(d)))
        ux, uy, uz = np.zeros(n), np.zeros(n), np.zeros(n)
        mk = np.zeros(n, dtype=np.uint64)
        si = np.zeros(n, dtype=np.uint32)
        anchors = np.zeros(3)
        self._check(self._lib.chui_treepm_dump_particles(self._h, n, ux.ctypes.data, uy.ctypes.data, uz.ctypes.data,
                                                         mk.ctypes.data, si.ctypes.data, anchors.ctypes.data))
        info = np.zeros(3, dtype=np.int32)
        self._check(self._lib.chui_treepm_tree_build_info(self._h, info.ctypes.data))
        r.update(ux=ux, uy=uy, uz=uz, morton_key=mk, sorted_index=si, anchors=anchors, n_nodes=nn,
                 unwrap_sorted_axes=int(info[0]), large_leaf=bool(info[1]), path_levels_retried=bool(info[2]))
        return r

    # -- KDK ------------------------------------------------------------------
    def kick(self, vx, vy, vz, ax, ay, az, kick_factor: float, drag_factor: float = 1.0, stream=None):
        arr = _Arrays(vx)
        if not arr.device:
            for v in (vx, vy, vz):
                if not (isinstance(v, np.ndarray) and v.dtype == np.float64 and v.flags.c_contiguous):
                    raise InvalidArgument(_abi.EINVAL, "kick updates contiguous float64 arrays in place")
        ps = [arr.ptr(a, np.float64) for a in (vx, vy, vz, ax, ay, az)]
        self._check(self._lib.chui_treepm_kick(self._h, len(vx), *[C.c_void_p(p) for p in ps], kick_factor,
                                               drag_factor, _abi.DEVICE if arr.device else _abi.HOST,
                                               C.c_void_p(stream) if stream else None))

    def drift(self, x, y, z, vx, vy, vz, drift_factor: float, stream=None):
        arr = _Arrays(x)
        if not arr.device:
            for v in (x, y, z):
                if not (isinstance(v, np.ndarray) and v.dtype == np.float64 and v.flags.c_contiguous):
                    raise InvalidArgument(_abi.EINVAL, "drift updates contiguous float64 arrays in place")
        ps = [arr.ptr(a, np.float64) for a in (x, y, z, vx, vy, vz)]
        self._check(self._lib.chui_treepm_drift(self._h, len(x), *[C.c_void_p(p) for p in ps], drift_factor,
                                                _abi.DEVICE if arr.device else _abi.HOST,
                                                C.c_void_p(stream) if stream else None))


def _adjoint_methods():
    """Reverse-mode entry points, attached to TreePmCoordinator below."""

    def force_vjp(self, x, y, z, mass, cot_x, cot_y, cot_z, uniform_mass: float = 0.0, softening=None):
        """J_a(x)^T cot for the full-set TreePM acceleration (chui_treepm_force_vjp;
        uniform softening only: a softening lane raises NotSupported)."""
        arr = _Arrays(x)
        src = _abi.Sources()
        src.count = len(x)
        src.x, src.y, src.z = arr.ptr(x, np.float64), arr.ptr(y, np.float64), arr.ptr(z, np.float64)
        src.mass = arr.ptr(mass, np.float64) if mass is not None else None
        src.uniform_mass = uniform_mass
        if softening is not None:
            src.softening = arr.ptr(softening, np.float64)
        cps = [arr.ptr(c, np.float64) for c in (cot_x, cot_y, cot_z)]
        outs = [arr.out(len(x), x) for _ in range(3)]
        st = _abi.Stats()
        self._check(self._lib.chui_treepm_force_vjp(self._h, C.byref(src), *[C.c_void_p(p) for p in cps],
                                                    *[C.c_void_p(o[1]) for o in outs],
                                                    _abi.DEVICE if arr.device else _abi.HOST, None, C.byref(st)))
        self.last_vjp_stats = st.as_dict()
        return tuple(o[0] for o in outs)

    def density_vjp(self, x, y, z, mass, rho_bar, uniform_mass: float = 0.0):
        """Transpose of assign_density for a flat cotangent grid (chui_pm_density_vjp)."""
        arr = _Arrays(x)
        src = _abi.Sources()
        src.count = len(x)
        src.x, src.y, src.z = arr.ptr(x, np.float64), arr.ptr(y, np.float64), arr.ptr(z, np.float64)
        src.mass = arr.ptr(mass, np.float64) if mass is not None else None
        src.uniform_mass = uniform_mass
        rb = arr.ptr(rho_bar, np.float64)
        outs = [arr.out(len(x), x) for _ in range(3)]
        self._check(self._lib.chui_pm_density_vjp(self._h, C.byref(src), C.c_void_p(rb),
                                                  *[C.c_void_p(o[1]) for o in outs],
                                                  _abi.DEVICE if arr.device else _abi.HOST, None))
        return tuple(o[0] for o in outs)

    def kdk_adjoint(self, gx, gy, gz, xb, yb, zb, vxb, vyb, vzb, axb, ayb, azb, drift, kick1, kick2, drag1, drag2,
                    first_step: bool, stream=None):
        """In-place transpose of one KDK step on CUDA float64 tensors (chui_treepm_kdk_adjoint)."""
        import torch
        ts = (gx, gy, gz, xb, yb, zb, vxb, vyb, vzb, axb, ayb, azb)
        for t in ts:
            if not (_is_torch(t) and t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
                raise InvalidArgument(_abi.EINVAL, "kdk_adjoint works in place on contiguous CUDA float64 tensors")
        self._check(self._lib.chui_treepm_kdk_adjoint(self._h, len(gx), *[C.c_void_p(t.data_ptr()) for t in ts],
                                                      drift, kick1, kick2, drag1, drag2, 1 if first_step else 0,
                                                      C.c_void_p(stream) if stream else None))

    def momentum_energy(self, mass, vx, vy, vz, ax=None, ay=None, az=None, uniform_mass: float = 0.0) -> dict:
        """FP64 global checks on the device: momentum, net force, kinetic energy, total mass."""
        arr = _Arrays(vx)
        mp = arr.ptr(mass, np.float64) if mass is not None else None
        vs = [arr.ptr(v, np.float64) for v in (vx, vy, vz)]
        acc = [arr.ptr(a, np.float64) if a is not None else None for a in (ax, ay, az)]
        out = np.zeros(8)
        self._check(self._lib.chui_treepm_momentum_energy(
            self._h, len(vx), C.c_void_p(mp) if mp else None, uniform_mass, *[C.c_void_p(p) for p in vs],
            *[C.c_void_p(p) if p else None for p in acc], _abi.DEVICE if arr.device else _abi.HOST, None,
            out.ctypes.data))
        return {"momentum": out[0:3].copy(), "net_force": out[3:6].copy(), "kinetic_energy": float(out[6]),
                "mass": float(out[7])}

    return force_vjp, density_vjp, kdk_adjoint, momentum_energy


(TreePmCoordinator.force_vjp, TreePmCoordinator.density_vjp, TreePmCoordinator.kdk_adjoint,
 TreePmCoordinator.momentum_energy) = _adjoint_methods()


def probe_fp32_peak_tflops(device: int = 0) -> float:
    """Measured FP32 FMA throughput of the GPU (the walk's roofline denominator)."""
    v = C.c_double()
    rc = _abi.load().chui_treepm_probe_fp32_peak(device, C.byref(v))
    if rc != 0:
        raise DeviceError(rc, "FP32 peak probe failed")
    return v.value


def kdk_factors_static(dt: float):
    """CosmologicalTimeline::prepareStep without a background: (D, K1, K2, drag1, drag2)."""
    f = np.zeros(5)
    rc = _abi.load().chui_treepm_kdk_factors_static(dt, f.ctypes.data)
    if rc != 0:
        raise InvalidArgument(rc, "dt must be finite and positive")
    return tuple(float(v) for v in f)


def kdk_factors_lcdm(scale_factor: float, dt: float, hubble_param: float = 0.674, omega_matter: float = 0.315,
                     omega_lambda: float = 0.685, omega_radiation: float = 0.0, omega_curvature: float = 0.0,
                     time_si_per_code: float = 3.0856775814913673e17) -> dict:
    """CosmologicalTimeline::prepareStep with a Lambda-CDM background
    (chui_treepm_kdk_factors_lcdm): the KDK factors of one step of dt (code
    time) from scale_factor. `factors` = (D, K1, K2, drag1, drag2) for the
    kick/drift calls; the rest are the source-kick factors and the midpoint
    and end scale factors."""
    class _Cosmo(C.Structure):
        _fields_ = [(k, C.c_double) for k in ("hubble_param", "omega_matter", "omega_lambda", "omega_radiation",
                                               "omega_curvature", "time_si_per_code")]
    c = _Cosmo(hubble_param, omega_matter, omega_lambda, omega_radiation, omega_curvature, time_si_per_code)
    f = np.zeros(10)
    rc = _abi.load().chui_treepm_kdk_factors_lcdm(C.byref(c), scale_factor, dt, f.ctypes.data)
    if rc == _abi.EINVAL:
        raise InvalidArgument(rc, "invalid background, scale factor or step")
    if rc != 0:
        raise OutOfRange(rc, "scale-factor advance could not be bracketed")
    keys = ("drift", "kick1", "kick2", "drag1", "drag2", "source_kick1", "source_kick2", "a_midpoint", "a_end",
            "drag")
    out = {k: float(v) for k, v in zip(keys, f)}
    out["factors"] = tuple(float(v) for v in f[:5])
    return out
