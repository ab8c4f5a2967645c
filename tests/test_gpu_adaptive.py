"""Adaptive-relative acceptance policy (TreePmOptions::acceptance_policy =
kAdaptiveRelative, internal/tree_pm_acceptance.hpp:53-139) on the GPU walks,
through the C-ABI, against the reference's own outputs (golden fixtures made
by tests/golden/make_golden.py) and the oracle.

Fixtures: a clustered box (lattice + 12 NFW halos, 19824 particles, mesh 32^3,
leaf 8, eps 0.01) with an acceleration history taken from the reference's
strict-policy solve of the same snapshot, some entries NaN / zero / below the
floor (the COM-distance fallback):
- adaptive_monopole: the production fast deck (relative monopole,
  COM-distance cutoff nodes, alpha 0.0025, maximum angle 1.0);
- adaptive_residual: residual-derivative estimator, contain nodes, alpha
  0.005, maximum angle 0.5, on an active subset of 5000 targets;
- group_walk, group_walk_active: the fast deck and relative monopole with
  contain nodes under the reference's group walk (one conservative walk per
  leaf of targets, Gaussian Hermite pair table), all targets / the subset.

Bars: FP64 accelerations to FP64 round-off with the reference's traversal
counters; mixed precision with the per-node walk: the reference's node
counters exactly (decisions are made in FP32 with a guard band and re-made in
FP64 where the band does not decide), pair counts within FP32 rounding of
r_cut; mixed accelerations median <= 1e-4, 99th percentile <= 1e-3.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import chui_treepm as ct  # noqa: E402
import oracle  # noqa: E402
from chui_treepm import ics  # noqa: E402
from conftest import golden_params, load_golden  # noqa: E402

pytestmark = pytest.mark.gpu

CASES = ["adaptive_monopole", "adaptive_residual"]
GROUP_CASES = ["group_walk", "group_walk_active"]
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
    policy, estimator, cutoff_policy = (int(v) for v in g["adaptive"])
    angle, rel_tol, floor = (float(v) for v in g["adaptive_f"])
    mesh = [int(v) for v in g["mesh"]]
    group_walk, lookup = (int(v) for v in g["group"]) if "group" in g else (0, 0)
    return ct.TreePmConfig(group_walk_enabled=group_walk, gaussian_pair_lookup=lookup,pm_grid_nx=mesh[0], pm_grid_ny=mesh[1], pm_grid_nz=mesh[2], box_x=float(g["box"][0]),
                           box_y=float(g["box"][1]), box_z=float(g["box"][2]), asmth_cells=asmth, rcut_cells=rcut,
                           opening_theta=theta, opening_criterion=criterion, multipole_order=order,
                           max_leaf_size=leaf, assignment_scheme=scheme, window_deconvolution=deconv,
                           gravitational_constant=gconst, softening=eps, precision=precision,
                           diagnostics=diagnostics, acceptance_policy=policy, adaptive_error_estimator=estimator,
                           cutoff_node_policy=cutoff_policy, adaptive_maximum_opening_angle=angle,
                           relative_force_tolerance=rel_tol, relative_force_acceleration_floor=floor)


def _active(g):
    return g["active"] if len(g["active"]) else None


def rel_err(got, ref):
    g = np.stack(got)
    r = np.stack(ref)
    den = np.linalg.norm(r, axis=0)
    scale = max(np.median(den), 1e-300)
    return np.linalg.norm(g - r, axis=0) / np.maximum(den, 1e-6 * scale)


@pytest.mark.parametrize("name", CASES + GROUP_CASES)
def test_fp64_adaptive_matches_reference(cuda_ok, name):
    g = load_golden(name)
    with ct.TreePmCoordinator(cfg_for(g, ct._abi.FP64)) as s:
        r = s.solve_active_set(g["x"], g["y"], g["z"], g["m"], active=_active(g),
                               previous_acceleration=g["prev_acc"])
    scale = np.abs(np.concatenate([g["ax"], g["ay"], g["az"]])).max()
    for k in ("ax", "ay", "az"):
        assert np.abs(r[k] - g[k]).max() <= 1e-9 * scale, k
    st = r["stats"]
    assert [st[k] for k in COUNTER_KEYS] == [int(v) for v in g["counters"]]


@pytest.mark.parametrize("name", CASES + GROUP_CASES)
def test_mixed_adaptive_matches_reference(cuda_ok, name):
    """Per-node mixed walk: the reference's decisions and forces. Production
    walk (subtree blocks replace some accepted multipoles by their exact
    pairs): at least as close to the strict FP64 forces as the reference's
    adaptive answer is."""
    g = load_golden(name)
    ref = dict(zip(COUNTER_KEYS, (int(v) for v in g["counters"])))
    with ct.TreePmCoordinator(cfg_for(g, ct._abi.MIXED, 1)) as s:
        r = s.solve_active_set(g["x"], g["y"], g["z"], g["m"], active=_active(g),
                               previous_acceleration=g["prev_acc"])
    e = rel_err([r["ax"], r["ay"], r["az"]], [g["ax"], g["ay"], g["az"]])
    assert np.median(e) <= 1e-4, np.median(e)
    assert np.percentile(e, 99) <= 1e-3, np.percentile(e, 99)
    st = r["stats"]
    assert [st[k] for k in NODE_KEYS] == [ref[k] for k in NODE_KEYS]
    assert abs(st["direct_pair_evaluations"] - ref["direct_pair_evaluations"]) <= \
        1e-6 * ref["direct_pair_evaluations"] + 2

    strict = cfg_for(g, ct._abi.FP64)
    strict.acceptance_policy = ct._abi.POLICY_STRICT
    strict.group_walk_enabled = strict.gaussian_pair_lookup = 0
    with ct.TreePmCoordinator(strict) as s:
        r64 = s.solve_active_set(g["x"], g["y"], g["z"], g["m"], active=_active(g))
    truth = [r64["ax"], r64["ay"], r64["az"]]
    with ct.TreePmCoordinator(cfg_for(g, ct._abi.MIXED, 0)) as s:
        rp = s.solve_active_set(g["x"], g["y"], g["z"], g["m"], active=_active(g),
                                previous_acceleration=g["prev_acc"])
    e_prod = rel_err([rp["ax"], rp["ay"], rp["az"]], truth)
    e_ref = rel_err([g["ax"], g["ay"], g["az"]], truth)
    assert np.median(e_prod) <= max(1e-4, 1.1 * np.median(e_ref)), (np.median(e_prod), np.median(e_ref))
    assert np.percentile(e_prod, 99) <= max(1e-3, 1.1 * np.percentile(e_ref, 99))


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("precision", [ct._abi.FP64, ct._abi.MIXED])
def test_adaptive_without_history_matches_oracle(cuda_ok, name, precision):
    """No history at all: every target takes the COM-distance fallback
    (with the adaptive envelope, containment and cutoff-node rules)."""
    g = load_golden(name)
    p = golden_params(g)
    o = oracle.treepm_solve(g["x"], g["y"], g["z"], g["m"], p, active=_active(g))
    with ct.TreePmCoordinator(cfg_for(g, precision)) as s:
        r = s.solve_active_set(g["x"], g["y"], g["z"], g["m"], active=_active(g))
    oc = o["counters"]
    want = {"visited_nodes": oc["visited"], "accepted_nodes": oc["accepted"], "opened_nodes": oc["opened"],
            "cutoff_pruned_nodes": oc["pruned"], "accepted_internal_multipoles": oc["multipoles"],
            "accepted_leaves": oc["leaves"]}
    st = r["stats"]
    assert {k: st[k] for k in NODE_KEYS} == want
    e = rel_err([r["ax"], r["ay"], r["az"]], [o["ax"], o["ay"], o["az"]])
    if precision == ct._abi.FP64:
        assert e.max() <= 1e-9, e.max()
    else:
        assert np.median(e) <= 1e-4 and np.percentile(e, 99) <= 1e-3, (np.median(e), np.percentile(e, 99))


def test_strict_relative_criterion_with_history(cuda_ok):
    """The strict policy's relative-force MAC with history
    (acceptNodeByMac, internal/tree_interaction_common.hpp:45-75) against the
    oracle, whose adaptive and strict walks are pinned to the reference."""
    g = load_golden("adaptive_monopole")
    p = golden_params(g)
    p.policy = 0
    p.criterion = 2
    prev = g["prev_acc"]
    o = oracle.treepm_solve(g["x"], g["y"], g["z"], g["m"], p, prev_acc=prev)
    for precision in (ct._abi.FP64, ct._abi.MIXED):
        cfg = cfg_for(g, precision)
        cfg.acceptance_policy = ct._abi.POLICY_STRICT
        cfg.opening_criterion = ct._abi.OPEN_RELATIVE
        with ct.TreePmCoordinator(cfg) as s:
            r = s.solve_active_set(g["x"], g["y"], g["z"], g["m"], previous_acceleration=prev)
        st = r["stats"]
        assert st["accepted_internal_multipoles"] == o["counters"]["multipoles"]
        assert st["visited_nodes"] == o["counters"]["visited"]
        e = rel_err([r["ax"], r["ay"], r["az"]], [o["ax"], o["ay"], o["az"]])
        assert np.median(e) <= (1e-12 if precision == ct._abi.FP64 else 1e-4)


@pytest.mark.parametrize("estimator,cutoff_policy,angle,alpha", [
    (ct._abi.ESTIMATOR_RELATIVE_MONOPOLE, ct._abi.CUTOFF_COM_DISTANCE, 1.0, 0.0025),
    (ct._abi.ESTIMATOR_RESIDUAL_DERIVATIVE, ct._abi.CUTOFF_CONTAIN_NODE, 0.5, 0.005)])
def test_adaptive_clustered_64(cuda_ok, estimator, cutoff_policy, angle, alpha):
    """Clustered 64^3 box (262144 particles, L = 50, 120 NFW halos over 3
    decades, mesh 64^3, leaf 16, eps 0.002) with a same-snapshot history from
    the strict FP64 solve: mixed per-node walk node counters equal the FP64
    walk's and its forces meet the mixed bar against it; the production walk
    is at least as close to the strict FP64 forces as the FP64 adaptive walk."""
    n_side, box = 64, 50.0
    x, y, z, *_ = ics.clustered_box(n_side ** 3, box, 0.6, 120, 3.0, 0.5, 11)
    m = np.full(len(x), 1.0 / len(x))
    base = dict(pm_grid_nx=n_side, pm_grid_ny=n_side, pm_grid_nz=n_side, box_x=box, box_y=box, box_z=box,
                opening_theta=0.5, max_leaf_size=16, softening=0.002)
    with ct.TreePmCoordinator(ct.TreePmConfig(**base, precision=ct._abi.FP64, diagnostics=1)) as s:
        r0 = s.solve_active_set(x, y, z, m)
    prev = np.sqrt(r0["ax"] ** 2 + r0["ay"] ** 2 + r0["az"] ** 2)
    adaptive = dict(acceptance_policy=ct._abi.POLICY_ADAPTIVE, adaptive_error_estimator=estimator,
                    cutoff_node_policy=cutoff_policy, adaptive_maximum_opening_angle=angle,
                    relative_force_tolerance=alpha)
    out = {}
    for key, prec, diag in (("fp64", ct._abi.FP64, 1), ("mixed", ct._abi.MIXED, 1), ("prod", ct._abi.MIXED, 0)):
        with ct.TreePmCoordinator(ct.TreePmConfig(**base, **adaptive, precision=prec, diagnostics=diag)) as s:
            r = s.solve_active_set(x, y, z, m, previous_acceleration=prev)
            out[key] = ([r[k] for k in ("ax", "ay", "az")], dict(r["stats"]))
    ref, st64 = out["fp64"]
    assert st64["accepted_internal_multipoles"] > 0
    e = rel_err(out["mixed"][0], ref)
    assert np.median(e) <= 1e-4 and np.percentile(e, 99) <= 1e-3, (np.median(e), np.percentile(e, 99))
    # production walk: at least as close to the strict FP64 forces as the FP64 adaptive walk
    truth = [r0["ax"], r0["ay"], r0["az"]]
    e_prod = rel_err(out["prod"][0], truth)
    e_ada = rel_err(ref, truth)
    assert np.median(e_prod) <= max(1e-4, 1.1 * np.median(e_ada)), (np.median(e_prod), np.median(e_ada))
    assert np.percentile(e_prod, 99) <= max(1e-3, 1.1 * np.percentile(e_ada, 99))
    assert [out["mixed"][1][k] for k in NODE_KEYS] == [st64[k] for k in NODE_KEYS]
    pairs = st64["direct_pair_evaluations"]
    assert abs(out["mixed"][1]["direct_pair_evaluations"] - pairs) <= 1e-6 * pairs
    # the adaptive policy's purpose: fewer pairs than the strict walk of the same state
    assert pairs < r0["stats"]["direct_pair_evaluations"]


@pytest.mark.parametrize("cutoff_policy", [ct._abi.CUTOFF_COM_DISTANCE, ct._abi.CUTOFF_CONTAIN_NODE])
def test_group_walk_clustered_64(cuda_ok, cutoff_policy):
    """Clustered 64^3 box under the group walk (fast deck settings): the mixed
    walk's node counters equal the FP64 group walk's (groups decided in FP64 by
    one lane per group in each warp), its forces meet the mixed bar against
    it, and the production walk is at least as close to the strict FP64 forces
    as the FP64 group walk."""
    n_side, box = 64, 50.0
    x, y, z, *_ = ics.clustered_box(n_side ** 3, box, 0.6, 120, 3.0, 0.5, 11)
    m = np.full(len(x), 1.0 / len(x))
    base = dict(pm_grid_nx=n_side, pm_grid_ny=n_side, pm_grid_nz=n_side, box_x=box, box_y=box, box_z=box,
                opening_theta=0.5, max_leaf_size=16, softening=0.002)
    with ct.TreePmCoordinator(ct.TreePmConfig(**base, precision=ct._abi.FP64, diagnostics=1)) as s:
        r0 = s.solve_active_set(x, y, z, m)
    prev = np.sqrt(r0["ax"] ** 2 + r0["ay"] ** 2 + r0["az"] ** 2)
    prev[::97] = np.nan  # some groups fall back to per-target walks
    group = dict(acceptance_policy=ct._abi.POLICY_ADAPTIVE, adaptive_error_estimator=ct._abi.ESTIMATOR_RELATIVE_MONOPOLE,
                 cutoff_node_policy=cutoff_policy, adaptive_maximum_opening_angle=1.0, relative_force_tolerance=0.0025,
                 group_walk_enabled=1, gaussian_pair_lookup=1)
    out = {}
    for key, prec, diag in (("fp64", ct._abi.FP64, 1), ("mixed", ct._abi.MIXED, 1), ("prod", ct._abi.MIXED, 0)):
        with ct.TreePmCoordinator(ct.TreePmConfig(**base, **group, precision=prec, diagnostics=diag)) as s:
            r = s.solve_active_set(x, y, z, m, previous_acceleration=prev)
            out[key] = ([r[k] for k in ("ax", "ay", "az")], dict(r["stats"]))
    ref, st64 = out["fp64"]
    assert st64["accepted_internal_multipoles"] > 0
    e = rel_err(out["mixed"][0], ref)
    assert np.median(e) <= 1e-4 and np.percentile(e, 99) <= 1e-3, (np.median(e), np.percentile(e, 99))
    assert [out["mixed"][1][k] for k in NODE_KEYS] == [st64[k] for k in NODE_KEYS]
    pairs = st64["direct_pair_evaluations"]
    assert abs(out["mixed"][1]["direct_pair_evaluations"] - pairs) <= 1e-6 * pairs
    truth = [r0["ax"], r0["ay"], r0["az"]]
    e_prod = rel_err(out["prod"][0], truth)
    e_grp = rel_err(ref, truth)
    assert np.median(e_prod) <= max(1e-4, 1.1 * np.median(e_grp)), (np.median(e_prod), np.median(e_grp))
    assert np.percentile(e_prod, 99) <= max(1e-3, 1.1 * np.percentile(e_grp, 99))
