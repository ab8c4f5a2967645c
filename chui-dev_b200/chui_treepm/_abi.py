"""ctypes binding of the C-ABI in include/chui_treepm.h.

The shared library is chui-dev_b200/_build/libchui_treepm.so, built by
chui-dev_b200/Makefile (or __graft_entry__.build()). There is no CPU
fallback: if the library is missing, loading fails with an error.
"""
from __future__ import annotations

import ctypes as C
import os

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "_build", "libchui_treepm.so")

OK, EINVAL, ERANGE, ENOMEM, ESTATE, EDEVICE, ENOTSUP = 0, 22, 34, 12, 71, 5, 95
HOST, DEVICE = 0, 1
MIXED, FP64 = 0, 1
CIC, TSC = 0, 1
OPEN_GEOMETRIC, OPEN_COM_DISTANCE, OPEN_RELATIVE = 0, 1, 2
POLICY_STRICT, POLICY_ADAPTIVE = 0, 1
ESTIMATOR_RESIDUAL_DERIVATIVE, ESTIMATOR_RELATIVE_MONOPOLE = 0, 1
CUTOFF_CONTAIN_NODE, CUTOFF_COM_DISTANCE = 0, 1
BOUNDARY_PERIODIC, BOUNDARY_ISOLATED_OPEN = 0, 1


class Config(C.Structure):
    _fields_ = [
        ("pm_grid_nx", C.c_int64), ("pm_grid_ny", C.c_int64), ("pm_grid_nz", C.c_int64),
        ("box_x", C.c_double), ("box_y", C.c_double), ("box_z", C.c_double),
        ("asmth_cells", C.c_double), ("rcut_cells", C.c_double), ("opening_theta", C.c_double),
        ("opening_criterion", C.c_int32), ("multipole_order", C.c_int32),
        ("max_leaf_size", C.c_int64),
        ("assignment_scheme", C.c_int32), ("window_deconvolution", C.c_int32),
        ("gravitational_constant", C.c_double), ("softening", C.c_double),
        ("acceptance_policy", C.c_int32), ("precision", C.c_int32), ("device", C.c_int32),
        ("diagnostics", C.c_int32),
        ("adaptive_error_estimator", C.c_int32), ("cutoff_node_policy", C.c_int32),
        ("adaptive_maximum_opening_angle", C.c_double), ("relative_force_tolerance", C.c_double),
        ("relative_force_acceleration_floor", C.c_double),
        ("group_walk_enabled", C.c_int32), ("gaussian_pair_lookup", C.c_int32),
        ("boundary_condition", C.c_int32), ("short_range_only", C.c_int32),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("visited_nodes", C.c_uint64), ("accepted_nodes", C.c_uint64), ("opened_nodes", C.c_uint64),
        ("direct_pair_evaluations", C.c_uint64), ("cutoff_pruned_nodes", C.c_uint64),
        ("cutoff_skipped_pairs", C.c_uint64), ("accepted_internal_multipoles", C.c_uint64),
        ("accepted_leaves", C.c_uint64), ("node_count", C.c_uint64), ("maximum_depth", C.c_uint32),
        ("path_words", C.c_uint32), ("pm_ms", C.c_double), ("tree_build_ms", C.c_double),
        ("walk_ms", C.c_double), ("total_ms", C.c_double), ("kernel_launches", C.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


DP = C.POINTER(C.c_double)
U32P = C.POINTER(C.c_uint32)


class Sources(C.Structure):
    _fields_ = [("count", C.c_int64), ("x", C.c_void_p), ("y", C.c_void_p), ("z", C.c_void_p),
                ("mass", C.c_void_p), ("uniform_mass", C.c_double), ("softening", C.c_void_p)]


class Accumulator(C.Structure):
    _fields_ = [("active_count", C.c_int64), ("active_index", C.c_void_p),
                ("accel_x", C.c_void_p), ("accel_y", C.c_void_p), ("accel_z", C.c_void_p),
                ("target_x", C.c_void_p), ("target_y", C.c_void_p), ("target_z", C.c_void_p),
                ("long_range_x", C.c_void_p), ("long_range_y", C.c_void_p), ("long_range_z", C.c_void_p),
                ("short_range_x", C.c_void_p), ("short_range_y", C.c_void_p), ("short_range_z", C.c_void_p),
                ("nearest_pair_r2", C.c_void_p), ("previous_acceleration_magnitude", C.c_void_p),
                ("target_softening", C.c_void_p)]


class TreeDump(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in (
        "center_x", "center_y", "center_z", "half_size", "mass", "com_x", "com_y", "com_z",
        "quad_xx", "quad_xy", "quad_xz", "quad_yy", "quad_yz", "quad_zz", "second_moment_trace",
        "child_count", "child_index", "particle_begin", "particle_count")]


# Every entry point declared in include/chui_treepm.h (checked by tests).
EXPORTED = (
    "chui_treepm_config_default", "chui_treepm_create", "chui_treepm_destroy",
    "chui_treepm_set_config", "chui_treepm_last_error", "chui_treepm_solve",
    "chui_pm_assign_density", "chui_pm_cells", "chui_treepm_tree_node_count",
    "chui_treepm_dump_tree", "chui_treepm_tree_build_info", "chui_treepm_dump_particles", "chui_treepm_kick", "chui_treepm_drift",
    "chui_treepm_kdk_factors_static", "chui_treepm_kdk_factors_lcdm", "chui_treepm_probe_fp32_peak", "chui_pm_assign_density_static",
    "chui_treepm_force_vjp", "chui_pm_density_vjp", "chui_treepm_kdk_adjoint", "chui_treepm_momentum_energy",
)
STATIC_MAX_CELLS = 262144  # CHUI_PM_STATIC_MAX_CELLS

_lib = None


def load(path: str | None = None):
    """Load the C-ABI library (fails loudly when it has not been built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.isfile(p):
        raise FileNotFoundError(
            f"B200 TreePM library not built: {p} (run `make -C chui-dev_b200` or __graft_entry__.build())")
    L = C.CDLL(p)
    vp = C.c_void_p
    L.chui_treepm_config_default.argtypes = [C.POINTER(Config)]
    L.chui_treepm_create.argtypes = [C.POINTER(Config), C.POINTER(vp)]
    L.chui_treepm_destroy.argtypes = [vp]
    L.chui_treepm_destroy.restype = None
    L.chui_treepm_set_config.argtypes = [vp, C.POINTER(Config)]
    L.chui_treepm_last_error.argtypes = [vp]
    L.chui_treepm_last_error.restype = C.c_char_p
    L.chui_treepm_solve.argtypes = [vp, C.POINTER(Sources), C.POINTER(Accumulator), C.c_int, C.c_int, vp,
                                    C.POINTER(Stats)]
    L.chui_treepm_solve_visit_range.argtypes = [vp, C.POINTER(Sources), C.POINTER(Accumulator), C.c_int, C.c_int,
                                                vp, C.POINTER(Stats), C.c_int64, C.c_int64]
    L.chui_treepm_visit_order.argtypes = [vp, C.c_int64, C.c_int64, vp, C.c_int, vp]
    L.chui_treepm_walk_cost.argtypes = [vp, C.c_int64, C.c_int64, vp, C.c_int, vp]
    L.chui_pm_assign_density.argtypes = [vp, C.POINTER(Sources), vp, C.c_int, vp]
    L.chui_pm_cells.argtypes = [vp, C.POINTER(Sources), vp, C.c_int, vp]
    L.chui_treepm_tree_node_count.argtypes = [vp, C.POINTER(C.c_int64)]
    L.chui_treepm_dump_tree.argtypes = [vp, C.POINTER(TreeDump)]
    L.chui_treepm_dump_particles.argtypes = [vp, C.c_int64, vp, vp, vp, vp, vp, vp]
    L.chui_treepm_tree_build_info.argtypes = [vp, vp]
    L.chui_treepm_kick.argtypes = [vp, C.c_int64, vp, vp, vp, vp, vp, vp, C.c_double, C.c_double, C.c_int, vp]
    L.chui_treepm_drift.argtypes = [vp, C.c_int64, vp, vp, vp, vp, vp, vp, C.c_double, C.c_int, vp]
    L.chui_treepm_kdk_factors_static.argtypes = [C.c_double, vp]
    L.chui_treepm_kdk_factors_lcdm.argtypes = [vp, C.c_double, C.c_double, vp]
    L.chui_treepm_probe_fp32_peak.argtypes = [C.c_int, C.POINTER(C.c_double)]
    L.chui_pm_assign_density_static.argtypes = [C.POINTER(Config), C.POINTER(Sources), vp, C.c_int, vp]
    L.chui_treepm_force_vjp.argtypes = [vp, C.POINTER(Sources), vp, vp, vp, vp, vp, vp, C.c_int, vp,
                                        C.POINTER(Stats)]
    L.chui_pm_density_vjp.argtypes = [vp, C.POINTER(Sources), vp, vp, vp, vp, C.c_int, vp]
    L.chui_treepm_kdk_adjoint.argtypes = [vp, C.c_int64] + [vp] * 12 + [C.c_double] * 5 + [C.c_int, vp]
    L.chui_treepm_momentum_energy.argtypes = [vp, C.c_int64, vp, C.c_double] + [vp] * 6 + [C.c_int, vp, vp]
    for name in EXPORTED:
        fn = getattr(L, name)
        if fn.restype is C.c_int or name not in ("chui_treepm_destroy", "chui_treepm_last_error"):
            if name not in ("chui_treepm_destroy", "chui_treepm_last_error"):
                fn.restype = C.c_int
    if path is None:
        _lib = L
    return L
