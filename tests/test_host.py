"""Host-side checks that need no GPU: the C-ABI library exports every entry
point include/chui_treepm.h declares, the `.param.txt` knob mapping, the
synthetic IC generators and the FP32 kernel polynomial."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import chui_treepm as ct
from chui_treepm import _abi, ics

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names += re.findall(r"\b(chui_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    lib = _abi.load()
    names = declared_functions()
    assert len(names) >= 14
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_abi.EXPORTED) | (set(names) - set(_abi.EXPORTED))


def test_config_defaults_match_reference_defaults():
    c = _abi.Config()
    assert _abi.load().chui_treepm_config_default(c) == 0
    assert (c.pm_grid_nx, c.asmth_cells, c.rcut_cells, c.opening_theta, c.max_leaf_size) == (16, 1.25, 6.25, 0.7, 16)
    assert c.opening_criterion == _abi.OPEN_COM_DISTANCE and c.multipole_order == 2
    # TreePmOptions / TreeGravityOptions defaults (tree_pm_coupling.hpp:243-332, tree_gravity.hpp:30-43)
    assert c.acceptance_policy == _abi.POLICY_STRICT
    assert c.adaptive_error_estimator == _abi.ESTIMATOR_RESIDUAL_DERIVATIVE
    assert c.cutoff_node_policy == _abi.CUTOFF_CONTAIN_NODE
    assert (c.adaptive_maximum_opening_angle, c.relative_force_tolerance,
            c.relative_force_acceleration_floor) == (0.25, 0.005, 1e-30)
    assert c.group_walk_enabled == 0 and c.gaussian_pair_lookup == 0
    assert c.boundary_condition == _abi.BOUNDARY_PERIODIC
    # the Python mirror carries the same defaults
    py = ct.TreePmConfig().to_c()
    for name, _ in _abi.Config._fields_:
        if name not in ("pm_grid_nx", "pm_grid_ny", "pm_grid_nz", "box_x", "box_y", "box_z", "window_deconvolution",
                        "diagnostics"):
            assert getattr(py, name) == getattr(c, name), name


@pytest.mark.parametrize("field,value", [("adaptive_maximum_opening_angle", 1.5),
                                         ("adaptive_maximum_opening_angle", 0.0),
                                         ("relative_force_tolerance", -1.0),
                                         ("relative_force_acceleration_floor", 0.0),
                                         ("acceptance_policy", 2), ("adaptive_error_estimator", 5),
                                         ("cutoff_node_policy", -1), ("boundary_condition", 2)])
def test_invalid_adaptive_options_are_rejected(field, value):
    # validateTreePmOptions (tree_pm_coupling.cpp:300-340) runs before any device work
    c = _abi.Config()
    lib = _abi.load()
    lib.chui_treepm_config_default(c)
    setattr(c, field, value)
    h = C.c_void_p()
    assert lib.chui_treepm_create(C.byref(c), C.byref(h)) == _abi.EINVAL


def test_kdk_static_factors():
    assert ct.kdk_factors_static(0.2) == (0.2, 0.1, 0.1, 1.0, 1.0)
    with pytest.raises(ValueError):
        ct.kdk_factors_static(-1.0)


DECK = """
schema_version = 1
[cosmology]
box_size_x = 20 mpc
box_size_y = 20 mpc
box_size_z = 20 mpc
[numerics]
gravity_softening = 15 kpc
treepm_pm_grid_nx = 32
treepm_pm_grid_ny = 32
treepm_pm_grid_nz = 32
treepm_asmth_cells = 1.25
treepm_rcut_cells = 6.25
treepm_tree_opening_criterion = geometric
treepm_tree_opening_theta = 0.6
treepm_tree_max_leaf_size = 32
treepm_assignment_scheme = cic
treepm_enable_window_deconvolution = false
"""


def test_param_deck_mapping():
    c = ct.config_from_param_text(DECK)
    assert (c.pm_grid_nx, c.box_x, c.opening_theta, c.max_leaf_size) == (32, 20.0, 0.6, 32)
    assert c.opening_criterion == _abi.OPEN_GEOMETRIC and c.assignment_scheme == _abi.CIC
    assert c.window_deconvolution == 0
    assert abs(c.softening - 0.015) < 1e-15
    assert abs(c.mesh_spacing - 20.0 / 32) < 1e-12
    with pytest.raises(ValueError):
        ct.config_from_param_text(DECK.replace("geometric", "bogus"))
    assert c.acceptance_policy == _abi.POLICY_STRICT


FAST_DECK = DECK + """treepm_adaptive_acceptance_enabled = true
treepm_adaptive_error_estimator = relative_monopole
treepm_cutoff_node_policy = com_distance
treepm_adaptive_maximum_opening_angle = 1.0
treepm_tree_relative_force_tolerance = 0.0025
treepm_group_walk_enabled = true
treepm_gaussian_pair_lookup_enabled = true
"""


def test_param_deck_adaptive_keys():
    c = ct.config_from_param_text(FAST_DECK)
    assert c.acceptance_policy == _abi.POLICY_ADAPTIVE
    assert c.adaptive_error_estimator == _abi.ESTIMATOR_RELATIVE_MONOPOLE
    assert c.cutoff_node_policy == _abi.CUTOFF_COM_DISTANCE
    assert (c.adaptive_maximum_opening_angle, c.relative_force_tolerance) == (1.0, 0.0025)
    assert c.relative_force_acceleration_floor == 1e-30
    assert c.group_walk_enabled == 1 and c.gaussian_pair_lookup == 1
    with pytest.raises(ValueError):
        ct.config_from_param_text(FAST_DECK.replace("relative_monopole", "bogus"))
    with pytest.raises(ValueError):
        ct.config_from_param_text(FAST_DECK.replace("= com_distance", "= bogus"))


def test_zeldovich_lattice_statistics():
    x, y, z, vx, vy, vz = ics.zeldovich_lattice(16, 10.0, 0.2, seed=5)
    assert len(x) == 16 ** 3 and x.min() >= 0 and x.max() < 10.0
    spacing = 10.0 / 16
    rms = np.sqrt(np.mean(vx ** 2 + vy ** 2 + vz ** 2))
    assert abs(rms - 0.2 * spacing) < 1e-9
    x2, *_ = ics.zeldovich_lattice(16, 10.0, 0.2, seed=5)
    assert np.array_equal(x, x2)


def test_clustered_box_counts():
    x, y, z, vx, vy, vz = ics.clustered_box(20000, 100.0, 0.4, 30, 3.0, 0.5, seed=2)
    assert len(x) == 20000
    assert np.all((x >= 0) & (x < 100.0)) and np.all((z >= 0) & (z < 100.0))


def test_fp32_kernel_polynomial_accuracy():
    """The per-configuration fit of H(t) = L(q)/q^3 (the Gaussian long-range
    coefficient of tree_pm_split_kernel.hpp:109-128): the pair kernel's
    9-term form is accurate to 5e-5, the 12-term form (multipole
    derivatives) to 1e-6, at the default r_cut / r_s = 5."""
    from scipy.special import erf
    t_cut = (6.25 / 2.5) ** 2
    t = np.linspace(1e-3, t_cut, 1000)
    q = np.sqrt(t)
    h_ref = (erf(q) - 2 * q * np.exp(-t) / np.sqrt(np.pi)) / (t * q)
    # same construction as the library: Chebyshev interpolation on [0, t_cut]
    for m, tol in ((9, 5e-5), (12, 1e-6)):
        k = np.arange(m)
        xk = np.cos(np.pi * (k + 0.5) / m)
        tk = (xk + 1) * 0.5 * t_cut
        qk = np.sqrt(tk)
        fk = (erf(qk) - 2 * qk * np.exp(-tk) / np.sqrt(np.pi)) / (tk * qk)
        cheb = np.polynomial.chebyshev.chebfit(xk, fk, m - 1)
        approx = np.polynomial.chebyshev.chebval(2 * t / t_cut - 1, cheb)
        assert np.max(np.abs(approx - h_ref) / h_ref) < tol, m


def test_isolated_boundary_validation():
    """Isolated/open PM (pm_solver.cpp:1664-1667, :5069-5071): no window
    deconvolution, at least 3 cells per axis; the periodic cutoff limit does
    not apply."""
    lib = _abi.load()
    for field, value, text in (("window_deconvolution", 1, "window deconvolution"),
                               ("pm_grid_nz", 2, "nx,ny,nz >= 3")):
        c = _abi.Config()
        lib.chui_treepm_config_default(c)
        c.boundary_condition = _abi.BOUNDARY_ISOLATED_OPEN
        setattr(c, field, value)
        h = C.c_void_p()
        assert lib.chui_treepm_create(C.byref(c), C.byref(h)) == _abi.EINVAL, field
        assert text in lib.chui_treepm_last_error(None).decode()
    deck = DECK + "[mode]\ngravity_boundary = isolated_monopole\n"
    assert ct.config_from_param_text(deck).boundary_condition == _abi.BOUNDARY_ISOLATED_OPEN
    deck = DECK + "[mode]\nmode = isolated_galaxy\n"
    assert ct.config_from_param_text(deck).boundary_condition == _abi.BOUNDARY_ISOLATED_OPEN
    deck = DECK + "[mode]\nmode = cosmo_cube\n"
    assert ct.config_from_param_text(deck).boundary_condition == _abi.BOUNDARY_PERIODIC
    with pytest.raises(ValueError):
        ct.config_from_param_text(DECK + "[mode]\ngravity_boundary = open\n")


def test_cpp_shim_compiles_and_links(tmp_path):
    """The C++20 shim (the class a CHUI build compiles in place of the
    reference's TreePmCoordinator) and its example program build against the
    C-ABI header and link against the library; running it needs a GPU
    (tests/test_gpu_cpp_shim.py)."""
    import shutil
    import subprocess
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    host = os.path.join(ROOT, "chui-dev_b200", "host")
    build = os.path.dirname(_abi.LIB_PATH)
    exe = tmp_path / "shim_example"
    subprocess.run(["g++", "-std=c++20", "-O1", "-Wall", "-Werror", os.path.join(host, "shim_example.cpp"),
                    f"-L{build}", "-lchui_treepm", "-o", str(exe)], check=True)
    assert exe.exists()


def test_cosmosim_adapter_compiles_against_the_reference_headers(tmp_path):
    """The coordinator over the reference's own types
    (chui-dev_b200/host/cosmosim_tree_pm_coordinator.hpp) and an example that
    calls solveActiveSetWithPmCadence the way GravityRuntimeImpl does
    (gravity_runtime.cpp:2383-2424) compile against the reference's headers,
    warning-free in their own code, and link against libchui_treepm.so alone.
    Needs the reference checkout (CHUI_REFERENCE); running it needs a GPU
    (tests/test_gpu_cpp_shim.py)."""
    import shutil
    import subprocess
    import sys
    sys.path.insert(0, ROOT)
    import __graft_entry__ as ge
    ref = os.environ.get("CHUI_REFERENCE", ge.REFERENCE)
    if shutil.which("g++") is None or not os.path.isfile(
            os.path.join(ref, "include", "cosmosim", "gravity", "tree_pm_coupling.hpp")):
        pytest.skip("reference headers not present")
    exe = tmp_path / "cosmosim_example"
    r = subprocess.run(ge.cosmosim_example_command(ref, str(exe)), capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    own = [ln for ln in r.stderr.splitlines() if "warning" in ln and "chui-dev_b200/host" in ln]
    assert not own, own
    assert exe.exists()


def test_lcdm_kdk_factors_match_reference():
    """chui_treepm_kdk_factors_lcdm against the reference's
    CosmologicalTimeline::prepareStep (tests/golden/kdk_factors.npz, from the
    reference built here): three backgrounds, scale factors 0.02-1, steps
    1e-6-0.05."""
    g = np.load(os.path.join(ROOT, "tests", "golden", "kdk_factors.npz"))
    for row, ref in zip(g["inputs"], g["factors"]):
        h, om, ol, orad, ok, tspc, a, dt = (float(v) for v in row)
        f = ct.kdk_factors_lcdm(a, dt, hubble_param=h, omega_matter=om, omega_lambda=ol, omega_radiation=orad,
                                omega_curvature=ok, time_si_per_code=tspc)
        got = [f[k] for k in ("drift", "kick1", "kick2", "drag1", "drag2", "source_kick1", "source_kick2",
                              "a_midpoint", "a_end", "drag")]
        np.testing.assert_allclose(got, ref, rtol=1e-13, atol=0.0)
    with pytest.raises(ct.InvalidArgument):
        ct.kdk_factors_lcdm(0.5, 0.01, omega_matter=0.3, omega_lambda=0.6)  # densities do not sum to 1
    with pytest.raises(ct.InvalidArgument):
        ct.kdk_factors_lcdm(-1.0, 0.01)
