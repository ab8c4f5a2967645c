"""Test infrastructure (oracle): ctypes binding of the C restatement
(oracle/treepm_oracle.c, built into oracle/_lib/libchui_oracle.so by
oracle/Makefile). Used only by tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline arm as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libchui_oracle.so")


class Params(C.Structure):
    _fields_ = [
        ("box", C.c_double * 3),
        ("mesh", C.c_int64 * 3),
        ("asmth_cells", C.c_double),
        ("rcut_cells", C.c_double),
        ("theta", C.c_double),
        ("G", C.c_double),
        ("epsilon", C.c_double),
        ("leaf_size", C.c_int64),
        ("scheme", C.c_int32),
        ("deconvolution", C.c_int32),
        ("criterion", C.c_int32),
        ("quadrupole", C.c_int32),
        ("policy", C.c_int32),
        ("estimator", C.c_int32),
        ("cutoff_policy", C.c_int32),
        ("reserved", C.c_int32),
        ("adaptive_angle", C.c_double),
        ("rel_tol", C.c_double),
        ("accel_floor", C.c_double),
        ("group_walk", C.c_int32),
        ("gaussian_lookup", C.c_int32),
        ("boundary", C.c_int32),
        ("reserved2", C.c_int32),
    ]


class Counters(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in
                ("visited", "accepted", "opened", "pairs", "pruned", "pair_skips", "multipoles", "leaves")]


def make_params(box=(1.0, 1.0, 1.0), mesh=(16, 16, 16), asmth=1.25, rcut=6.25, theta=0.5, g=1.0,
                eps=0.0, leaf=16, scheme=0, deconv=0, criterion=1, quadrupole=1, policy=0, estimator=0,
                cutoff_policy=0, adaptive_angle=0.25, rel_tol=0.005, accel_floor=1e-30, group_walk=0,
                gaussian_lookup=0, boundary=0) -> Params:
    """Defaults are TreePmOptions' (include/cosmosim/gravity/tree_pm_coupling.hpp:243-332):
    strict-reference policy; the adaptive fields apply with policy=1 (estimator 0 residual
    derivative / 1 relative monopole, cutoff_policy 0 contain node / 1 COM distance)."""
    p = Params()
    p.box = (C.c_double * 3)(*box)
    p.mesh = (C.c_int64 * 3)(*mesh)
    p.asmth_cells = asmth
    p.rcut_cells = rcut
    p.theta = theta
    p.G = g
    p.epsilon = eps
    p.leaf_size = leaf
    p.scheme = scheme
    p.deconvolution = deconv
    p.criterion = criterion
    p.quadrupole = quadrupole
    p.policy = policy
    p.estimator = estimator
    p.cutoff_policy = cutoff_policy
    p.adaptive_angle = adaptive_angle
    p.rel_tol = rel_tol
    p.accel_floor = accel_floor
    p.group_walk = group_walk
    p.gaussian_lookup = gaussian_lookup
    p.boundary = boundary
    return p


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-f", os.path.join("oracle", "Makefile")],
                   cwd=os.path.dirname(HERE), check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.isfile(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        dp = C.POINTER(C.c_double)
        L.oracle_treepm_solve.restype = C.c_int
        L.oracle_treepm_solve2.restype = C.c_int
        L.oracle_tree_build.restype = C.c_void_p
        L.oracle_tree_build.argtypes = [C.c_int64, dp, dp, dp, dp, C.POINTER(Params), C.POINTER(C.c_int)]
        L.oracle_tree_node_count.restype = C.c_int64
        L.oracle_tree_node_count.argtypes = [C.c_void_p]
        L.oracle_tree_max_depth.restype = C.c_uint32
        L.oracle_tree_max_depth.argtypes = [C.c_void_p]
        L.oracle_tree_copy.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.oracle_tree_free.argtypes = [C.c_void_p]
        L.oracle_unwrap_axis.restype = C.c_double
        L.oracle_unwrap_axis.argtypes = [C.c_int64, dp, C.c_double, C.c_int, dp]
        L.oracle_mesh_spacing.restype = C.c_double
        for fn in ("oracle_long_range_factor", "oracle_short_range_factor"):
            getattr(L, fn).restype = C.c_double
            getattr(L, fn).argtypes = [C.c_double, C.c_double]
        L.oracle_residual_inv_r3.restype = C.c_double
        L.oracle_residual_inv_r3.argtypes = [C.c_double, C.c_double, C.c_double]
        _lib = L
    return _lib


def _p(a, ct=C.c_double):
    return a.ctypes.data_as(C.POINTER(ct))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def treepm_solve(x, y, z, m, params: Params, active=None, prev_acc=None) -> dict:
    """prev_acc: per active target |a_previous| (the acceleration history of the
    relative criteria), or None for no history."""
    x, y, z, m = _f64(x), _f64(y), _f64(z), _f64(m)
    n = len(x)
    act = None if active is None else np.ascontiguousarray(active, dtype=np.uint32)
    na = n if act is None else len(act)
    prev = None if prev_acc is None else _f64(prev_acc)
    if prev is not None and len(prev) != na:
        raise ValueError("prev_acc needs one entry per active target")
    out = {k: np.zeros(na) for k in ("ax", "ay", "az", "pm_ax", "pm_ay", "pm_az",
                                      "tree_ax", "tree_ay", "tree_az", "nearest_r2")}
    cnt = Counters()
    rc = lib().oracle_treepm_solve2(
        C.c_int64(n), _p(x), _p(y), _p(z), _p(m), C.c_int64(na),
        None if act is None else _p(act, C.c_uint32), C.byref(params), None if prev is None else _p(prev),
        *[_p(out[k]) for k in ("ax", "ay", "az", "pm_ax", "pm_ay", "pm_az",
                               "tree_ax", "tree_ay", "tree_az", "nearest_r2")],
        C.byref(cnt))
    if rc != 0:
        raise RuntimeError(f"oracle_treepm_solve failed with status {rc}")
    out["counters"] = {k: int(getattr(cnt, k)) for k, _ in Counters._fields_}
    return out


def pm_density(x, y, z, m, params: Params) -> np.ndarray:
    x, y, z, m = _f64(x), _f64(y), _f64(z), _f64(m)
    cells = int(params.mesh[0] * params.mesh[1] * params.mesh[2])
    rho = np.zeros(cells)
    lib().oracle_pm_density(C.c_int64(len(x)), _p(x), _p(y), _p(z), _p(m), C.byref(params), _p(rho))
    return rho


def pm_cells(x, y, z, params: Params) -> np.ndarray:
    x, y, z = _f64(x), _f64(y), _f64(z)
    out = np.zeros(3 * len(x), dtype=np.int64)
    lib().oracle_pm_cells(C.c_int64(len(x)), _p(x), _p(y), _p(z), C.byref(params), _p(out, C.c_int64))
    return out.reshape(-1, 3)


def pm_force_grids(x, y, z, m, params: Params):
    x, y, z, m = _f64(x), _f64(y), _f64(z), _f64(m)
    cells = int(params.mesh[0] * params.mesh[1] * params.mesh[2])
    f = [np.zeros(cells) for _ in range(3)]
    lib().oracle_pm_force_grids(C.c_int64(len(x)), _p(x), _p(y), _p(z), _p(m), C.byref(params),
                                _p(f[0]), _p(f[1]), _p(f[2]))
    return f


def pm_interpolate(params: Params, fx, fy, fz, tx, ty, tz):
    tx, ty, tz = _f64(tx), _f64(ty), _f64(tz)
    a = [np.zeros(len(tx)) for _ in range(3)]
    lib().oracle_pm_interpolate(C.byref(params), _p(_f64(fx)), _p(_f64(fy)), _p(_f64(fz)),
                                C.c_int64(len(tx)), _p(tx), _p(ty), _p(tz), _p(a[0]), _p(a[1]), _p(a[2]))
    return a


def unwrap_axis(x, box: float, canonical: bool):
    x = _f64(x)
    out = np.zeros_like(x)
    anchor = lib().oracle_unwrap_axis(len(x), _p(x), box, 1 if canonical else 0, _p(out))
    return out, anchor


def tree_build(ux, uy, uz, m, params: Params) -> dict:
    ux, uy, uz, m = _f64(ux), _f64(uy), _f64(uz), _f64(m)
    n = len(ux)
    st = C.c_int(0)
    h = lib().oracle_tree_build(n, _p(ux), _p(uy), _p(uz), _p(m), C.byref(params), C.byref(st))
    try:
        if st.value != 0:
            raise RuntimeError(f"oracle tree build failed with status {st.value}")
        nn = lib().oracle_tree_node_count(h)
        r = {"n_nodes": nn, "max_depth": lib().oracle_tree_max_depth(h)}
        r["morton_key"] = np.zeros(n, dtype=np.uint64)
        lib().oracle_tree_copy(h, 0, r["morton_key"].ctypes.data)
        r["sorted_index"] = np.zeros(n, dtype=np.uint32)
        lib().oracle_tree_copy(h, 1, r["sorted_index"].ctypes.data)
        names = ("center_x", "center_y", "center_z", "half", "mass", "com_x", "com_y", "com_z",
                 "qxx", "qxy", "qxz", "qyy", "qyz", "qzz", "trace")
        for i, k in enumerate(names):
            r[k] = np.zeros(nn)
            lib().oracle_tree_copy(h, 2 + i, r[k].ctypes.data)
        for fid, k, cnt in ((17, "child_count", nn), (18, "child_index", 8 * nn),
                            (19, "particle_begin", nn), (20, "particle_count", nn)):
            r[k] = np.zeros(cnt, dtype=np.uint32)
            lib().oracle_tree_copy(h, fid, r[k].ctypes.data)
        return r
    finally:
        lib().oracle_tree_free(h)


def kick(vx, vy, vz, ax, ay, az, kick_factor: float, drag: float) -> None:
    lib().oracle_kick(C.c_int64(len(vx)), _p(vx), _p(vy), _p(vz), _p(_f64(ax)), _p(_f64(ay)), _p(_f64(az)),
                      C.c_double(kick_factor), C.c_double(drag))


def drift(x, y, z, vx, vy, vz, drift_factor: float, box) -> None:
    b = (C.c_double * 3)(*box)
    lib().oracle_drift(C.c_int64(len(x)), _p(x), _p(y), _p(z), _p(_f64(vx)), _p(_f64(vy)), _p(_f64(vz)),
                       C.c_double(drift_factor), b)
