"""Per-particle softening on the GPU against the reference's own solve with a
TreeSofteningView (tests/golden/softening_*.npz, made by
tests/golden/make_golden.py): source epsilons by override mask (some masks
off: the configured epsilon), mixed-softening nodes under the envelope guard,
and an active subset with target sidecars. The view is resolved into the
C-ABI's epsilon lanes by chui_treepm.softening.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import chui_treepm as ct  # noqa: E402
from conftest import load_golden  # noqa: E402
from test_gpu_parity import COUNTER_KEYS, cfg_for, rel_err  # noqa: E402

pytestmark = pytest.mark.gpu

CASES = ["softening_mixed", "softening_active"]
NODE_KEYS = ("visited_nodes", "accepted_nodes", "opened_nodes", "cutoff_pruned_nodes",
             "accepted_internal_multipoles", "accepted_leaves")


@pytest.fixture(scope="module")
def cuda_ok():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True


def lanes(g):
    n = len(g["x"])
    eps0 = float(g["params"][4])
    src = ct.softening.resolve_sources(n, eps0, epsilon=g["src_eps"], override_mask=g["src_mask"])
    act = g["active"] if len(g["active"]) else None
    tgt = None
    if "tgt_eps" in g:
        tgt = ct.softening.resolve_targets(act, src, n, eps0, epsilon=g["tgt_eps"], override_mask=g["tgt_mask"])
    return act, src, tgt


@pytest.mark.parametrize("name", CASES)
def test_fp64_softening_matches_reference(cuda_ok, name):
    """The per-node FP64 walk: forces to FP64 round-off and every traversal
    counter equal to the reference's."""
    g = load_golden(name)
    act, src, tgt = lanes(g)
    with ct.TreePmCoordinator(cfg_for(g, ct._abi.FP64)) as s:
        r = s.solve_active_set(g["x"], g["y"], g["z"], g["m"], active=act, softening=src, target_softening=tgt,
                               nearest_pair=act is None)
    scale = np.abs(np.concatenate([g["ax"], g["ay"], g["az"]])).max()
    for k in ("ax", "ay", "az"):
        assert np.abs(r[k] - g[k]).max() <= 1e-9 * scale, k
    assert [r["stats"][k] for k in COUNTER_KEYS] == [int(v) for v in g["counters"]]
    if act is None:
        fin = np.isfinite(g["nearest_r2"])
        np.testing.assert_allclose(r["nearest_r2"][fin], g["nearest_r2"][fin], rtol=1e-12)


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("diagnostics", [1, 0])
def test_mixed_softening_matches_reference(cuda_ok, name, diagnostics):
    """Mixed precision: the force bar against the reference; with diagnostics
    the node counters equal the reference's (pairs within FP32 rounding of
    r_cut)."""
    g = load_golden(name)
    act, src, tgt = lanes(g)
    cfg = cfg_for(g, ct._abi.MIXED)
    cfg.diagnostics = diagnostics
    with ct.TreePmCoordinator(cfg) as s:
        r = s.solve_active_set(g["x"], g["y"], g["z"], g["m"], active=act, softening=src, target_softening=tgt)
    e = rel_err([r["ax"], r["ay"], r["az"]], [g["ax"], g["ay"], g["az"]])
    print(f"{name} diagnostics={diagnostics}: median {np.median(e):.2e} p99 {np.percentile(e, 99):.2e}")
    assert np.median(e) <= 1e-4, np.median(e)
    assert np.percentile(e, 99) <= 1e-3, np.percentile(e, 99)
    if diagnostics:
        ref = dict(zip(COUNTER_KEYS, (int(v) for v in g["counters"])))
        assert [r["stats"][k] for k in NODE_KEYS] == [ref[k] for k in NODE_KEYS]
        assert abs(r["stats"]["direct_pair_evaluations"] - ref["direct_pair_evaluations"]) <= \
            1e-5 * ref["direct_pair_evaluations"]


def test_softening_lane_changes_the_answer(cuda_ok):
    """The lanes reach the walk: the same state with uniform softening differs
    from the reference's per-particle answer by far more than the bar."""
    g = load_golden("softening_mixed")
    with ct.TreePmCoordinator(cfg_for(g, ct._abi.FP64)) as s:
        r = s.solve_active_set(g["x"], g["y"], g["z"], g["m"])
    e = rel_err([r["ax"], r["ay"], r["az"]], [g["ax"], g["ay"], g["az"]])
    assert np.percentile(e, 99) > 1e-3


def test_softening_lane_errors(cuda_ok):
    g = load_golden("softening_mixed")
    n = len(g["x"])
    bad = np.full(n, 0.01)
    bad[7] = -1.0
    with ct.TreePmCoordinator(cfg_for(g, ct._abi.MIXED)) as s:
        with pytest.raises(ct.InvalidArgument, match="finite non-negative"):
            s.solve_active_set(g["x"], g["y"], g["z"], g["m"], softening=bad)
        # independent targets with a source lane need their own lane
        with pytest.raises(ct.InvalidArgument, match="target-owned softening"):
            s.solve_active_set(g["x"], g["y"], g["z"], g["m"], softening=np.full(n, 0.01),
                               targets=(g["x"][:10], g["y"][:10], g["z"][:10]))
        with pytest.raises(ct.NotSupported):
            s.force_vjp(g["x"], g["y"], g["z"], g["m"], *(np.zeros(n) for _ in range(3)), softening=np.full(n, 0.01))
