"""Isolated/open boundaries (PmBoundaryCondition::kIsolatedOpen) through the
C-ABI against the reference's own outputs (tests/golden/make_golden.py): the
zero-padded PM with the split Green function -erf(r / 2 r_s) / r and one-sided
boundary gradients (solvePoissonIsolatedOpen, pm_solver.cpp:4942-5337), the
non-periodic deposit and interpolation (particles outside [0, L) take no PM
force and deposit nothing), the tree on the caller's coordinates and the walk
without periodic images (tree_pm_coupling.cpp:3179-3196, 3560-3562).

Fixtures: a clustered distribution in the middle of a box of 10 with
particles on and beyond the faces, mesh 16^3 (padded 32^3), leaf 8:
isolated_cic (all targets, unsoftened) and isolated_tsc_active (TSC, eps 0.02,
600 active targets). Bars as for the periodic path: FP64 to round-off with the
reference's counters, mixed median <= 1e-4 and 99th percentile <= 1e-3.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import chui_treepm as ct  # noqa: E402
import oracle  # noqa: E402
from conftest import golden_params, load_golden  # noqa: E402

pytestmark = pytest.mark.gpu

CASES = ["isolated_cic", "isolated_tsc_active"]
COUNTER_KEYS = ("visited_nodes", "accepted_nodes", "opened_nodes", "direct_pair_evaluations",
                "cutoff_pruned_nodes", "cutoff_skipped_pairs", "accepted_internal_multipoles", "accepted_leaves")
NODE_KEYS = ("visited_nodes", "accepted_nodes", "opened_nodes", "cutoff_pruned_nodes",
             "accepted_internal_multipoles", "accepted_leaves")


@pytest.fixture(scope="module")
def cuda_ok():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True


def cfg_for(g, precision, diagnostics=1):
    asmth, rcut, theta, gconst, eps = (float(v) for v in g["params"])
    leaf, scheme, deconv, criterion, order = (int(v) for v in g["iparams"])
    mesh = [int(v) for v in g["mesh"]]
    return ct.TreePmConfig(pm_grid_nx=mesh[0], pm_grid_ny=mesh[1], pm_grid_nz=mesh[2], box_x=float(g["box"][0]),
                           box_y=float(g["box"][1]), box_z=float(g["box"][2]), asmth_cells=asmth, rcut_cells=rcut,
                           opening_theta=theta, opening_criterion=criterion, multipole_order=order,
                           max_leaf_size=leaf, assignment_scheme=scheme, window_deconvolution=deconv,
                           gravitational_constant=gconst, softening=eps, precision=precision,
                           diagnostics=diagnostics, boundary_condition=ct._abi.BOUNDARY_ISOLATED_OPEN)


def _active(g):
    return g["active"] if len(g["active"]) else None


def rel_err(got, ref):
    g = np.stack(got)
    r = np.stack(ref)
    den = np.linalg.norm(r, axis=0)
    scale = max(np.median(den), 1e-300)
    return np.linalg.norm(g - r, axis=0) / np.maximum(den, 1e-6 * scale)


@pytest.mark.parametrize("name", CASES)
def test_fp64_isolated_matches_reference(cuda_ok, name):
    g = load_golden(name)
    act = _active(g)
    with ct.TreePmCoordinator(cfg_for(g, ct._abi.FP64)) as s:
        r = s.solve_active_set(g["x"], g["y"], g["z"], g["m"], active=act, long_range=True, short_range=True)
        t = s.dump_tree(len(g["x"]))
    for prefix in ("", "pm_"):
        ref = np.concatenate([g[prefix + k] for k in ("ax", "ay", "az")])
        got = np.concatenate([r[prefix + k] for k in ("ax", "ay", "az")])
        assert np.abs(got - ref).max() <= 1e-9 * np.abs(ref).max(), prefix
    rows = act if act is not None else np.arange(len(g["x"]))
    ref = np.concatenate([g[k][rows] for k in ("tree_ax", "tree_ay", "tree_az")])
    got = np.concatenate([r[k][rows] for k in ("tree_ax", "tree_ay", "tree_az")])
    assert np.abs(got - ref).max() <= 1e-9 * np.abs(ref).max()
    st = r["stats"]
    assert [st[k] for k in COUNTER_KEYS] == [int(v) for v in g["counters"]]
    # the tree is built on the caller's coordinates, bit-exact
    assert np.array_equal(t["ux"], g["ux"]) and np.array_equal(t["morton_key"], g["morton_key"])
    assert np.array_equal(t["sorted_index"], g["sorted_index"])


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("diagnostics", [1, 0])
def test_mixed_isolated_matches_reference(cuda_ok, name, diagnostics):
    g = load_golden(name)
    with ct.TreePmCoordinator(cfg_for(g, ct._abi.MIXED, diagnostics)) as s:
        r = s.solve_active_set(g["x"], g["y"], g["z"], g["m"], active=_active(g))
    e = rel_err([r["ax"], r["ay"], r["az"]], [g["ax"], g["ay"], g["az"]])
    assert np.median(e) <= 1e-4 and np.percentile(e, 99) <= 1e-3, (np.median(e), np.percentile(e, 99))
    if diagnostics:
        ref = dict(zip(COUNTER_KEYS, (int(v) for v in g["counters"])))
        assert [r["stats"][k] for k in NODE_KEYS] == [ref[k] for k in NODE_KEYS]


def test_isolated_density_matches_oracle(cuda_ok):
    g = load_golden("isolated_cic")
    p = golden_params(g)
    want = oracle.pm_density(g["x"], g["y"], g["z"], g["m"], p)
    for precision in (ct._abi.FP64, ct._abi.MIXED):
        with ct.TreePmCoordinator(cfg_for(g, precision)) as s:
            rho = s.assign_density(g["x"], g["y"], g["z"], g["m"])
        rho = rho.cpu().numpy() if hasattr(rho, "cpu") else np.asarray(rho)
        np.testing.assert_allclose(rho, want, rtol=0, atol=1e-12 * np.abs(want).max())


def test_isolated_adjoint_is_not_supported(cuda_ok):
    g = load_golden("isolated_cic")
    cot = [np.ones(len(g["x"]))] * 3
    with ct.TreePmCoordinator(cfg_for(g, ct._abi.FP64)) as s:
        with pytest.raises(ct.NotSupported):
            s.force_vjp(g["x"], g["y"], g["z"], g["m"], *cot)
