"""CUDA path against the reference's golden outputs and the oracle, through the
C-ABI (chui_treepm -> libchui_treepm.so).

Bars (as the build specification states them):
- Morton keys, sort order, CIC cell indices, leaf membership: bit-exact.
- FP64 GPU accelerations: the reference's values to FP64 round-off, with the
  same traversal counters.
- Mixed precision accelerations: median |da|/|a| <= 1e-4, 99th percentile
  <= 1e-3 against the reference.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import chui_treepm as ct  # noqa: E402
import oracle  # noqa: E402
from conftest import golden_params, load_golden  # noqa: E402

pytestmark = pytest.mark.gpu

# clustered64k_*: the headline settings (CIC with window deconvolution, theta
# 0.6, leaf 16) and the large configuration's tree (theta 0.7, leaf 32) on a
# clustered periodic box of 64000 particles
CASES = ["lattice16_cic", "clustered_tsc", "rect_active", "two_body", "quasi24", "duplicates", "config32",
         "clustered64k_cic", "clustered64k_t07_leaf32"]
COUNTER_KEYS = ("visited_nodes", "accepted_nodes", "opened_nodes", "direct_pair_evaluations",
                "cutoff_pruned_nodes", "cutoff_skipped_pairs", "accepted_internal_multipoles", "accepted_leaves")


def cfg_for(g, precision):
    asmth, rcut, theta, gconst, eps = (float(v) for v in g["params"])
    leaf, scheme, deconv, criterion, order = (int(v) for v in g["iparams"])
    mesh = [int(v) for v in g["mesh"]]
    return ct.TreePmConfig(pm_grid_nx=mesh[0], pm_grid_ny=mesh[1], pm_grid_nz=mesh[2], box_x=float(g["box"][0]),
                           box_y=float(g["box"][1]), box_z=float(g["box"][2]), asmth_cells=asmth, rcut_cells=rcut,
                           opening_theta=theta, opening_criterion=criterion, multipole_order=order,
                           max_leaf_size=leaf, assignment_scheme=scheme, window_deconvolution=deconv,
                           gravitational_constant=gconst, softening=eps, precision=precision, diagnostics=1)


def _active(g):
    return g["active"] if len(g["active"]) else None


def rel_err(got, ref):
    g = np.stack(got)
    r = np.stack(ref)
    den = np.linalg.norm(r, axis=0)
    scale = max(np.median(den), 1e-300)
    return np.linalg.norm(g - r, axis=0) / np.maximum(den, 1e-6 * scale)


@pytest.fixture(scope="module")
def cuda_ok():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("precision", [ct._abi.FP64, ct._abi.MIXED])
def test_tree_bit_exact(cuda_ok, name, precision):
    g = load_golden(name)
    with ct.TreePmCoordinator(cfg_for(g, precision)) as s:
        s.solve_active_set(g["x"], g["y"], g["z"], g["m"], active=_active(g))
        t = s.dump_tree(len(g["x"]))
    for a, key in enumerate(("ux", "uy", "uz")):
        assert np.array_equal(t[key], g[key]), key
    assert np.array_equal(t["anchors"], g["anchors"])
    assert t["n_nodes"] == len(g["half"])
    assert np.array_equal(t["morton_key"], g["morton_key"])
    assert np.array_equal(t["sorted_index"], g["sorted_index"])
    for k in ("particle_begin", "particle_count", "child_count", "child_index"):
        assert np.array_equal(t[k], g[k]), k
    for mine, ref in (("center_x", "center_x"), ("center_y", "center_y"), ("center_z", "center_z"),
                      ("half_size", "half")):
        assert np.array_equal(t[mine], g[ref]), mine
    np.testing.assert_allclose(t["mass"], g["mass"], rtol=1e-13, atol=1e-14 * g["mass"].max())
    for mine, ref in (("com_x", "com_x"), ("com_y", "com_y"), ("com_z", "com_z")):
        np.testing.assert_allclose(t[mine], g[ref], rtol=1e-13, atol=1e-13 * np.abs(g[ref]).max())
    qs = max(np.abs(g["trace"]).max(), 1e-300)
    for mine, ref in (("quad_xx", "qxx"), ("quad_xy", "qxy"), ("quad_zz", "qzz"), ("second_moment_trace", "trace")):
        assert np.abs(t[mine] - g[ref]).max() <= 1e-11 * qs, mine


@pytest.mark.parametrize("name", CASES)
def test_fp64_matches_reference(cuda_ok, name):
    g = load_golden(name)
    act = _active(g)
    with ct.TreePmCoordinator(cfg_for(g, ct._abi.FP64)) as s:
        r = s.solve_active_set(g["x"], g["y"], g["z"], g["m"], active=act, long_range=True, short_range=True,
                               nearest_pair=True)
    scale = np.abs(np.concatenate([g["ax"], g["ay"], g["az"]])).max()
    for k in ("ax", "ay", "az"):
        assert np.abs(r[k] - g[k]).max() <= 1e-9 * scale, k
    pscale = np.abs(np.concatenate([g["pm_ax"], g["pm_ay"], g["pm_az"]])).max()
    for k in ("pm_ax", "pm_ay", "pm_az"):
        assert np.abs(r[k] - g[k]).max() <= 1e-9 * pscale, k
    rows = act if act is not None else np.arange(len(g["x"]))
    for k in ("tree_ax", "tree_ay", "tree_az"):
        assert np.abs(r[k][rows] - g[k][rows]).max() <= 1e-9 * scale, k
    near = g["nearest_r2"][rows]
    fin = np.isfinite(near)
    assert np.array_equal(np.isfinite(r["nearest_r2"][rows]), fin)
    np.testing.assert_allclose(r["nearest_r2"][rows][fin], near[fin], rtol=1e-12)
    st = r["stats"]
    assert [st[k] for k in COUNTER_KEYS] == [int(v) for v in g["counters"]]


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("diagnostics", [1, 0])
def test_mixed_precision_matches_reference(cuda_ok, name, diagnostics):
    """diagnostics=0 is the production walk (subtree blocks, no counters)."""
    g = load_golden(name)
    act = _active(g)
    cfg = cfg_for(g, ct._abi.MIXED)
    cfg.diagnostics = diagnostics
    with ct.TreePmCoordinator(cfg) as s:
        r = s.solve_active_set(g["x"], g["y"], g["z"], g["m"], active=act)
    e = rel_err([r["ax"], r["ay"], r["az"]], [g["ax"], g["ay"], g["az"]])
    assert np.median(e) <= 1e-4, np.median(e)
    assert np.percentile(e, 99) <= 1e-3, np.percentile(e, 99)


@pytest.mark.parametrize("n_side,halos", [(48, 60), (64, 120)])
def test_production_walk_matches_diagnostic_walk(cuda_ok, n_side, halos):
    """Clustered boxes where many opened nodes qualify as subtree blocks. The
    production walk's pair set is the per-node walk's, except that strict
    multipoles inside a block are summed as the pairs they stand for: against
    the FP64 production walk (the same pair set) it differs only by FP32
    arithmetic; against the per-node walk also by those multipoles'
    truncation; and against the reference-exact FP64 per-node walk it meets
    the mixed bar. The lanes compared are the tree-only residual forces, a
    fraction of the total force, so their relative FP32 error is larger than
    the total force's (the total's is median 2.5e-7, p99 2.9e-6 at 256^3):
    the bars here are 1e-5 at the median and 3e-4 at the 99th percentile."""
    from chui_treepm import ics
    box = 50.0
    x, y, z, *_ = ics.clustered_box(n_side ** 3, box, 0.6, halos, 3.0, 0.5, 7)
    m = np.full(len(x), 1.0 / len(x))
    res = {}
    for key, prec, diag in (("d1", ct._abi.MIXED, 1), ("d0", ct._abi.MIXED, 0), ("f64", ct._abi.FP64, 1),
                            ("f64p", ct._abi.FP64, 0)):
        cfg = ct.TreePmConfig(pm_grid_nx=n_side, pm_grid_ny=n_side, pm_grid_nz=n_side, box_x=box, box_y=box,
                              box_z=box, opening_theta=0.6, max_leaf_size=16, softening=0.002, precision=prec,
                              diagnostics=diag)
        with ct.TreePmCoordinator(cfg) as s:
            r = s.solve_active_set(x, y, z, m, short_range=True)
            res[key] = [r["tree_ax"], r["tree_ay"], r["tree_az"]]
    e_fp32 = rel_err(res["d0"], res["f64p"])
    assert np.median(e_fp32) <= 1e-5, np.median(e_fp32)
    assert np.percentile(e_fp32, 99) <= 3e-4, np.percentile(e_fp32, 99)
    e_blocks = rel_err(res["d0"], res["d1"])
    assert np.median(e_blocks) <= 1e-5, np.median(e_blocks)
    assert np.percentile(e_blocks, 99) <= 3e-4, np.percentile(e_blocks, 99)
    e64 = rel_err(res["d0"], res["f64"])
    assert np.median(e64) <= 1e-4, np.median(e64)
    assert np.percentile(e64, 99) <= 1e-3, np.percentile(e64, 99)


def test_cic_cells_and_density_bit_exact(cuda_ok):
    for name in ("lattice16_cic", "clustered_tsc", "rect_active"):
        g = load_golden(name)
        p = golden_params(g)
        with ct.TreePmCoordinator(cfg_for(g, ct._abi.FP64)) as s:
            cells = s.cells(g["x"], g["y"], g["z"])
            rho = s.assign_density(g["x"], g["y"], g["z"], g["m"])
        assert np.array_equal(cells, oracle.pm_cells(g["x"], g["y"], g["z"], p)), name
        np.testing.assert_allclose(rho, g["density"], rtol=0, atol=1e-12 * np.abs(g["density"]).max())


@pytest.mark.parametrize("name", ["lattice16_cic", "config32"])
def test_kdk_step_matches_reference(cuda_ok, name):
    g = load_golden(name)
    drift, k1, k2, d1, d2 = (float(v) for v in g["kdk_factors"])
    dev = torch.device("cuda:0")
    t = {k: torch.tensor(g[k], device=dev) for k in ("x", "y", "z", "m", "vx", "vy", "vz")}
    with ct.TreePmCoordinator(cfg_for(g, ct._abi.FP64)) as s:
        r = s.solve_active_set(t["x"], t["y"], t["z"], t["m"])
        s.kick(t["vx"], t["vy"], t["vz"], r["ax"], r["ay"], r["az"], k1, d1)
        s.drift(t["x"], t["y"], t["z"], t["vx"], t["vy"], t["vz"], drift)
        x = t["x"].cpu().numpy()
        np.testing.assert_allclose(x, g["kdk_x"], rtol=0, atol=1e-12 * float(g["box"][0]))
        r2 = s.solve_active_set(t["x"], t["y"], t["z"], t["m"])
        s.kick(t["vx"], t["vy"], t["vz"], r2["ax"], r2["ay"], r2["az"], k2, d2)
    vs = np.abs(g["kdk_vx"]).max()
    for k in ("vx", "vy", "vz"):
        assert np.abs(t[k].cpu().numpy() - g["kdk_" + k]).max() <= 1e-9 * vs, k


def test_device_and_host_paths_agree(cuda_ok):
    g = load_golden("clustered_tsc")
    dev = torch.device("cuda:0")
    with ct.TreePmCoordinator(cfg_for(g, ct._abi.MIXED)) as s:
        h = s.solve_active_set(g["x"], g["y"], g["z"], g["m"])
        d = s.solve_active_set(*(torch.tensor(g[k], device=dev) for k in ("x", "y", "z", "m")))
    # FP32 mesh atomics make runs differ at single-precision round-off
    for k in ("ax", "ay", "az"):
        np.testing.assert_allclose(d[k].cpu().numpy(), h[k], rtol=1e-5, atol=1e-6 * np.abs(h[k]).max())
    # caller-provided outputs (pinned host arrays, device tensors) receive the same forces
    with ct.TreePmCoordinator(cfg_for(g, ct._abi.FP64)) as s:
        ref = s.solve_active_set(g["x"], g["y"], g["z"], g["m"])
        pinned = [torch.empty(len(g["x"]), dtype=torch.float64).pin_memory().numpy() for _ in range(3)]
        r = s.solve_active_set(g["x"], g["y"], g["z"], g["m"], out=pinned)
        assert all(r[k] is a for k, a in zip(("ax", "ay", "az"), pinned))
        tens = [torch.empty(len(g["x"]), dtype=torch.float64, device=dev) for _ in range(3)]
        s.solve_active_set(*(torch.tensor(g[k], device=dev) for k in ("x", "y", "z", "m")), out=tens)
    # (FP64 mesh atomics: equal up to summation-order round-off)
    for k, a, t in zip(("ax", "ay", "az"), pinned, tens):
        np.testing.assert_allclose(a, ref[k], rtol=1e-12, atol=1e-12 * np.abs(ref[k]).max())
        np.testing.assert_allclose(t.cpu().numpy(), ref[k], rtol=1e-12, atol=1e-12 * np.abs(ref[k]).max())


def test_explicit_targets_match_oracle_walk(cuda_ok):
    """Explicit target positions without source identity (reference: active
    index UINT32_MAX, tree_pm_coupling.cpp:4459-4485) equal the FP64 solve at
    those positions up to the self-pair the identity-less walk keeps."""
    g = load_golden("lattice16_cic")
    rng = np.random.default_rng(3)
    tx, ty, tz = (rng.uniform(0, 10.0, 64) for _ in range(3))
    with ct.TreePmCoordinator(cfg_for(g, ct._abi.FP64)) as s:
        r = s.solve_active_set(g["x"], g["y"], g["z"], g["m"], targets=(tx, ty, tz))
    # the same targets appended as massless sources with identity
    x = np.concatenate([g["x"], tx])
    y = np.concatenate([g["y"], ty])
    z = np.concatenate([g["z"], tz])
    m = np.concatenate([g["m"], np.zeros(64)])
    p = golden_params(g)
    o = oracle.treepm_solve(x, y, z, m, p, active=np.arange(len(g["x"]), len(x), dtype=np.uint32))
    e = rel_err([r["ax"], r["ay"], r["az"]], [o["ax"], o["ay"], o["az"]])
    assert np.max(e) < 1e-9


def test_errors_follow_reference_semantics(cuda_ok):
    g = load_golden("lattice16_cic")
    cfg = cfg_for(g, ct._abi.MIXED)
    with ct.TreePmCoordinator(cfg) as s:
        bad = g["x"].copy()
        bad[5] = np.nan
        with pytest.raises(ValueError, match="finite"):
            s.solve_active_set(bad, g["y"], g["z"], g["m"])
        neg = g["m"].copy()
        neg[3] = -1.0
        with pytest.raises(ValueError, match="non-negative"):
            s.solve_active_set(g["x"], g["y"], g["z"], neg)
        with pytest.raises(IndexError, match="active index"):
            s.solve_active_set(g["x"], g["y"], g["z"], g["m"], active=np.array([0, len(g["x"])], dtype=np.uint32))
    with ct.TreePmCoordinator(cfg) as s2:
        with pytest.raises(RuntimeError, match="reuse"):
            s2.solve_active_set_with_pm_cadence(g["x"], g["y"], g["z"], g["m"], False)
        s2.solve_active_set(g["x"], g["y"], g["z"], g["m"])
        r = s2.solve_active_set_with_pm_cadence(g["x"], g["y"], g["z"], g["m"], False)
        assert np.isfinite(r["ax"]).all()
    big = cfg_for(g, ct._abi.MIXED)
    big.rcut_cells = 16.0
    with pytest.raises(ValueError, match="cutoff_radius_comoving"):
        ct.TreePmCoordinator(big)


def test_uniform_mass_lane_matches_explicit_masses(cuda_ok):
    g = load_golden("config32")
    with ct.TreePmCoordinator(cfg_for(g, ct._abi.MIXED)) as s:
        a = s.solve_active_set(g["x"], g["y"], g["z"], g["m"])
        b = s.solve_active_set(g["x"], g["y"], g["z"], None, uniform_mass=float(g["m"][0]))
    for k in ("ax", "ay", "az"):
        np.testing.assert_allclose(a[k], b[k], rtol=1e-5, atol=1e-6 * np.abs(a[k]).max())


@pytest.mark.parametrize("name", CASES)
def test_fp64_production_matches_reference(cuda_ok, name):
    """The production solver in FP64 (diagnostics off: the mixed walk's
    traversal and subtree blocks with FP64 pairs and multipoles). Subtree
    blocks sum as pairs what the reference may accept as a strict multipole,
    so it equals the reference to FP64 round-off where no multipole is
    accepted and otherwise within the quadrupole truncation error."""
    g = load_golden(name)
    act = _active(g)
    cfg = cfg_for(g, ct._abi.FP64)
    cfg.diagnostics = 0
    with ct.TreePmCoordinator(cfg) as s:
        r = s.solve_active_set(g["x"], g["y"], g["z"], g["m"], active=act)
    e = rel_err([r["ax"], r["ay"], r["az"]], [g["ax"], g["ay"], g["az"]])
    print(f"{name}: FP64 production vs reference median {np.median(e):.2e} p99 {np.percentile(e, 99):.2e} "
          f"max {e.max():.2e}")
    if int(g["counters"][6]) == 0:  # no accepted multipoles
        scale = np.abs(np.concatenate([g["ax"], g["ay"], g["az"]])).max()
        for k in ("ax", "ay", "az"):
            assert np.abs(r[k] - g[k]).max() <= 1e-9 * scale, k
    assert np.median(e) <= 1e-8, np.median(e)
    assert np.percentile(e, 99) <= 1e-5, np.percentile(e, 99)


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("precision", [ct._abi.MIXED, ct._abi.FP64])
def test_production_walk_nearest_pair_and_counters(cuda_ok, name, precision):
    """The production walk (diagnostics 0) fills a requested nearest-pair lane
    and, with diagnostics 2, reports its own traversal counters. Its pairs are
    every source inside r_cut of the target (subtree blocks also sum what the
    reference accepts as far multipoles), a superset of the reference's
    direct pairs: the nearest pair is the reference's, or nearer."""
    g = load_golden(name)
    act = _active(g)
    rows = act if act is not None else np.arange(len(g["x"]))
    near_ref = g["nearest_r2"][rows]
    for diagnostics in (0, 2):
        cfg = cfg_for(g, precision)
        cfg.diagnostics = diagnostics
        with ct.TreePmCoordinator(cfg) as s:
            r = s.solve_active_set(g["x"], g["y"], g["z"], g["m"], active=act, nearest_pair=True)
        near = r["nearest_r2"][rows]
        fin = np.isfinite(near_ref)
        assert np.isfinite(near[fin]).all()
        # mixed: r^2 from FP32 offsets in the warp's frame (absolute error
        # ~1e-7 of the frame's extent), so the closest pairs carry up to
        # ~1e-4 relative error; the lane feeds a timestep criterion
        # (FP64: offsets formed in the warp's frame, ~1e-16 of its extent)
        tol = 1e-3 if precision == ct._abi.MIXED else 1e-9
        assert (near[fin] <= near_ref[fin] * (1 + tol) + 1e-30).all()
        same = np.abs(near[fin] - near_ref[fin]) <= tol * near_ref[fin] + 1e-30
        assert same.mean() >= 0.99, same.mean()
        st = r["stats"]
        if diagnostics == 2:
            ref = dict(zip(COUNTER_KEYS, (int(v) for v in g["counters"])))
            assert st["direct_pair_evaluations"] >= 0.99 * ref["direct_pair_evaluations"]
            assert st["visited_nodes"] > 0  # (small trees may be one subtree block: no accepted nodes)
    # the lane comes back without being asked for a counted walk, and the
    # forces are the production walk's
    e = rel_err([r["ax"], r["ay"], r["az"]], [g["ax"], g["ay"], g["az"]])
    assert np.median(e) <= 1e-4 and np.percentile(e, 99) <= 1e-3


@pytest.mark.parametrize("name", ["lattice16_cic", "clustered64k_cic", "rect_active"])
def test_short_range_only_is_the_tree_part(cuda_ok, name):
    """TreePmOptions::short_range_only (the integrator's split operator): the
    solve returns the short-range residual alone -- the reference's
    source-indexed tree-only lanes -- with zero long-range lanes, and needs no
    PM field (a reuse request does not fail)."""
    g = load_golden(name)
    act = _active(g)
    rows = act if act is not None else np.arange(len(g["x"]))
    cfg = cfg_for(g, ct._abi.FP64)
    cfg.short_range_only = 1
    scale = np.abs(np.concatenate([g["tree_ax"][rows], g["tree_ay"][rows], g["tree_az"][rows]])).max()
    with ct.TreePmCoordinator(cfg) as s:
        for refresh in (False, True):
            r = s.solve_active_set_with_pm_cadence(g["x"], g["y"], g["z"], g["m"], refresh, active=act,
                                                   long_range=True)
            for k in ("x", "y", "z"):
                assert np.abs(r["a" + k] - g["tree_a" + k][rows]).max() <= 1e-9 * scale, k
                assert np.all(r["pm_a" + k] == 0.0)


def _forms_case(kind, seed=11):
    """Particle sets that take each form of the tree build: evenly spaced
    distinct x (the gap buckets could hide the largest gap, so the unwrap
    sorts that axis), 1500 coincident particles (one leaf above the in-place
    ordering limit at the depth limit), and a clustered set (neither)."""
    rng = np.random.default_rng(seed)
    if kind == "spaced_x":
        n = 4096
        x = (rng.permutation(n) + 0.5) / n
        y, z = rng.random(n), rng.random(n)
    elif kind == "large_leaf":
        p = rng.random(3)
        x = np.concatenate([np.full(1500, p[0]), rng.random(2000)])
        y = np.concatenate([np.full(1500, p[1]), rng.random(2000)])
        z = np.concatenate([np.full(1500, p[2]), rng.random(2000)])
    else:
        c = rng.random((40, 3))
        pts = (c[rng.integers(0, 40, 20000)] + 0.02 * rng.standard_normal((20000, 3))) % 1.0
        x, y, z = pts[:, 0].copy(), pts[:, 1].copy(), pts[:, 2].copy()
        x[:50] -= 1.0  # some coordinates outside [0, L): the canonical map applies
    m = np.full(len(x), 1.0 / len(x))
    return x, y, z, m


def _check_tree_against_oracle(t, x, y, z, m, p):
    u = []
    for a, v in enumerate((x, y, z)):
        ua, anchor = oracle.unwrap_axis(v, 1.0, bool(v.min() >= 0.0 and v.max() < 1.0))
        assert np.array_equal(t["u" + "xyz"[a]], ua), a
        assert t["anchors"][a] == anchor, a
        u.append(ua)
    o = oracle.tree_build(u[0], u[1], u[2], m, p)
    assert t["n_nodes"] == o["n_nodes"]
    for k in ("morton_key", "sorted_index", "particle_begin", "particle_count", "child_count", "child_index"):
        assert np.array_equal(t[k], o[k]), k
    assert np.array_equal(t["half_size"], o["half"])


@pytest.mark.parametrize("kind", ["spaced_x", "large_leaf", "clustered"])
@pytest.mark.parametrize("precision", [ct._abi.FP64, ct._abi.MIXED])
def test_tree_build_forms_match_oracle(cuda_ok, kind, precision):
    """Each form of the build gives the oracle's tree: the unwrap by gap
    buckets or by sorting, the in-place or global within-leaf order, and the
    path sort by the previous tree's levels, repeated with every level when
    the tree is deeper (a shallow set first), or kept (the same set again)."""
    x, y, z, m = _forms_case(kind)
    p = oracle.make_params(box=(1.0, 1.0, 1.0), mesh=(16, 16, 16), eps=0.01, leaf=16)
    cfg = ct.TreePmConfig(pm_grid_nx=16, pm_grid_ny=16, pm_grid_nz=16, box_x=1.0, box_y=1.0, box_z=1.0,
                          asmth_cells=1.25, rcut_cells=6.25, opening_theta=0.5, opening_criterion=1,
                          multipole_order=2, max_leaf_size=16, softening=0.01, precision=precision)
    rng = np.random.default_rng(5)
    shallow = rng.random((3, 24))  # a root and its octants: depth 1
    with ct.TreePmCoordinator(cfg) as s:
        s.solve_active_set(shallow[0], shallow[1], shallow[2], np.full(24, 1.0 / 24))
        assert s.dump_tree(24)["n_nodes"] <= 9
        trees = []
        for _ in range(2):
            s.solve_active_set(x, y, z, m)
            trees.append(s.dump_tree(len(x)))
    for t in trees:
        _check_tree_against_oracle(t, x, y, z, m, p)
        assert t["unwrap_sorted_axes"] == (1 if kind == "spaced_x" else 0)
        assert t["large_leaf"] == (kind == "large_leaf")
    # the shallow tree's levels do not resolve these trees; the repeat's own do
    assert trees[0]["path_levels_retried"] and not trees[1]["path_levels_retried"]
