"""`.param.txt` TreePM knobs -> TreePmConfig.

Reads the keys the reference's typed config defines for TreePM
(include/cosmosim/core/config.hpp:776-821, section [numerics]) and the box
lengths of [cosmology], with the mapping GravityRuntimeImpl applies
(src/workflows/gravity_runtime.cpp:469-608): softening in kpc -> Mpc
(x 1e-3), r_s = treepm_asmth_cells x mesh spacing, r_cut = treepm_rcut_cells x
spacing, spacing = cbrt(prod L_a / n_a). Unknown keys are ignored: a deck
carries many subsystems this solver does not own.
"""
from __future__ import annotations

import re

from . import _abi
from .solver import TreePmConfig

# G in Mpc (km/s)^2 / Msun for the reference's default unit system
# (length mpc, mass msun, velocity km_s).
G_MPC_KMS2_PER_MSUN = 4.300917270036279e-09

_CRITERIA = {"geometric": _abi.OPEN_GEOMETRIC, "com_distance": _abi.OPEN_COM_DISTANCE,
             "relative_force_error": _abi.OPEN_RELATIVE}
_SCHEMES = {"cic": _abi.CIC, "tsc": _abi.TSC}
_ESTIMATORS = {"residual_derivative": _abi.ESTIMATOR_RESIDUAL_DERIVATIVE,
               "relative_monopole": _abi.ESTIMATOR_RELATIVE_MONOPOLE}
_CUTOFF_POLICIES = {"contain": _abi.CUTOFF_CONTAIN_NODE, "com_distance": _abi.CUTOFF_COM_DISTANCE}


def _bool(v: str) -> bool:
    v = v.strip().lower()
    if v in ("true", "1", "yes", "on"):
        return True
    if v in ("false", "0", "no", "off"):
        return False
    raise ValueError(f"invalid boolean '{v}'")


def _length_mpc(v: str) -> float:
    m = re.fullmatch(r"\s*([-+0-9.eE]+)\s*([A-Za-z]*)\s*", v)
    if not m:
        raise ValueError(f"invalid length '{v}'")
    val, unit = float(m.group(1)), m.group(2).lower()
    scale = {"": 1.0, "mpc": 1.0, "kpc": 1.0e-3, "pc": 1.0e-6}.get(unit)
    if scale is None:
        raise ValueError(f"unsupported length unit '{unit}'")
    return val * scale


def parse_param_text(text: str) -> dict:
    """Sectioned `key = value` pairs: {"section.key": "value"}."""
    out: dict = {}
    section = ""
    for raw in text.splitlines():
        line = raw.split("#", 1)[0].strip()
        if not line:
            continue
        if line.startswith("[") and line.endswith("]"):
            section = line[1:-1].strip()
            continue
        if "=" not in line:
            continue
        k, v = line.split("=", 1)
        out[f"{section}.{k.strip()}" if section else k.strip()] = v.strip()
    return out


def config_from_param_text(text: str, precision: int = _abi.MIXED, device: int = 0,
                           gravitational_constant: float | None = None) -> TreePmConfig:
    kv = parse_param_text(text)
    c = TreePmConfig(precision=precision, device=device)

    def get(key, conv, default=None):
        v = kv.get(key)
        if v is None or v == "":
            return default
        return conv(v)

    c.pm_grid_nx = get("numerics.treepm_pm_grid_nx", int, get("numerics.treepm_pm_grid", int, 16))
    c.pm_grid_ny = get("numerics.treepm_pm_grid_ny", int, c.pm_grid_nx)
    c.pm_grid_nz = get("numerics.treepm_pm_grid_nz", int, c.pm_grid_nx)
    c.box_x = get("cosmology.box_size_x", _length_mpc, 1.0)
    c.box_y = get("cosmology.box_size_y", _length_mpc, c.box_x)
    c.box_z = get("cosmology.box_size_z", _length_mpc, c.box_x)
    c.asmth_cells = get("numerics.treepm_asmth_cells", float, 1.25)
    c.rcut_cells = get("numerics.treepm_rcut_cells", float, 6.25)
    c.opening_theta = get("numerics.treepm_tree_opening_theta", float, 0.7)
    crit = get("numerics.treepm_tree_opening_criterion", lambda v: v.strip().lower(), "com_distance")
    if crit not in _CRITERIA:
        raise ValueError(f"key 'numerics.treepm_tree_opening_criterion': invalid value '{crit}'")
    c.opening_criterion = _CRITERIA[crit]
    c.max_leaf_size = get("numerics.treepm_tree_max_leaf_size", int, 16)
    scheme = get("numerics.treepm_assignment_scheme", lambda v: v.strip().lower(), "tsc")
    if scheme not in _SCHEMES:
        raise ValueError(f"key 'numerics.treepm_assignment_scheme': invalid value '{scheme}'")
    c.assignment_scheme = _SCHEMES[scheme]
    c.window_deconvolution = 1 if get("numerics.treepm_enable_window_deconvolution", _bool, True) else 0
    c.relative_force_tolerance = get("numerics.treepm_tree_relative_force_tolerance", float, 0.005)
    c.relative_force_acceleration_floor = get("numerics.treepm_tree_relative_force_acceleration_floor", float, 1e-30)
    if get("numerics.treepm_adaptive_acceptance_enabled", _bool, False):
        c.acceptance_policy = _abi.POLICY_ADAPTIVE
    c.adaptive_maximum_opening_angle = get("numerics.treepm_adaptive_maximum_opening_angle", float, 0.25)
    est = get("numerics.treepm_adaptive_error_estimator", lambda v: v.strip().lower(), "residual_derivative")
    if est not in _ESTIMATORS:
        raise ValueError(f"key 'numerics.treepm_adaptive_error_estimator': invalid value '{est}'")
    c.adaptive_error_estimator = _ESTIMATORS[est]
    cut = get("numerics.treepm_cutoff_node_policy", lambda v: v.strip().lower(), "contain")
    if cut not in _CUTOFF_POLICIES:
        raise ValueError(f"key 'numerics.treepm_cutoff_node_policy': invalid value '{cut}'")
    c.cutoff_node_policy = _CUTOFF_POLICIES[cut]
    c.group_walk_enabled = 1 if get("numerics.treepm_group_walk_enabled", _bool, False) else 0
    # mode.gravity_boundary (config.cpp:1148-1160): periodic, isolated_monopole, or auto =
    # periodic for the cosmo_cube and zoom_in modes (:3437-3439), the default mode being zoom_in
    gb = get("mode.gravity_boundary", lambda v: v.strip().lower(), "auto")
    if gb not in ("auto", "periodic", "isolated_monopole"):
        raise ValueError(f"key 'mode.gravity_boundary': invalid value '{gb}'")
    mode = get("mode.mode", lambda v: v.strip().lower(), "zoom_in")
    periodic = gb == "periodic" or (gb == "auto" and mode in ("cosmo_cube", "zoom_in"))
    c.boundary_condition = _abi.BOUNDARY_PERIODIC if periodic else _abi.BOUNDARY_ISOLATED_OPEN
    c.gaussian_pair_lookup = 1 if get("numerics.treepm_gaussian_pair_lookup_enabled", _bool, False) else 0
    soft = kv.get("numerics.gravity_softening")
    if soft:
        # gravity_softening_kpc_comoving * 1e-3 (gravity_runtime.cpp:579-581)
        c.softening = _length_mpc(soft if re.search(r"[A-Za-z]", soft) else soft + " kpc")
    else:
        c.softening = 1.0e-3
    c.gravitational_constant = gravitational_constant if gravitational_constant is not None else G_MPC_KMS2_PER_MSUN
    return c


def config_from_param_file(path: str, **kw) -> TreePmConfig:
    with open(path) as f:
        return config_from_param_text(f.read(), **kw)
