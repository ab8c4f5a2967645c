"""Mixed precision against the FP64 walk on the clustered 128^3 box (2.1M
particles, L = 100, 40 % of the mass in 300 NFW halos over 3 decades, the
rest a Zel'dovich lattice of 0.5 spacing rms; mesh 128^3, leaf 16), at both
opening angles the clustered case is quoted at. The production walk
(diagnostics off) and the per-node walk must both meet the force bar, and
the FP64 walk's node counters must equal the mixed per-node walk's. The mixed
walk tests each pair against r_cut in FP32, so pairs within FP32 rounding of
r_cut may be counted differently (a few in 1e10)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import chui_treepm as ct  # noqa: E402
from chui_treepm import ics  # noqa: E402

pytestmark = pytest.mark.gpu

NODE_COUNTERS = ("visited_nodes", "accepted_nodes", "opened_nodes", "cutoff_pruned_nodes",
                 "accepted_internal_multipoles", "accepted_leaves")


@pytest.fixture(scope="module")
def box128():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    x, y, z, *_ = ics.clustered_box(128 ** 3, 100.0, 0.4, 300, 3.0, 0.5, 42)
    m = np.full(len(x), 1.0 / len(x))
    return [torch.tensor(v, device="cuda") for v in (x, y, z, m)]


def rel_err(a, b):
    d = np.sqrt(sum((a[k] - b[k]) ** 2 for k in range(3)))
    n = np.sqrt(sum(b[k] ** 2 for k in range(3)))
    return d / np.maximum(n, 1e-300)


@pytest.mark.parametrize("theta", [0.5, 0.7])
def test_mixed_matches_fp64_on_clustered_128(box128, theta):
    out = {}
    for key, prec, diag in (("fp64", ct._abi.FP64, 1), ("mixed", ct._abi.MIXED, 1), ("prod", ct._abi.MIXED, 0)):
        cfg = ct.TreePmConfig(pm_grid_nx=128, pm_grid_ny=128, pm_grid_nz=128, box_x=100.0, box_y=100.0,
                              box_z=100.0, opening_theta=theta, max_leaf_size=16, softening=0.001,
                              precision=prec, diagnostics=diag)
        with ct.TreePmCoordinator(cfg) as s:
            r = s.solve_active_set(*box128)
            out[key] = ([r[k].cpu().numpy() for k in ("ax", "ay", "az")], dict(s.last_stats))
    ref = out["fp64"][0]
    for key in ("mixed", "prod"):
        e = rel_err(out[key][0], ref)
        assert np.median(e) <= 1e-4 and np.percentile(e, 99) <= 1e-3, (key, np.median(e), np.percentile(e, 99))
    assert [out["mixed"][1][k] for k in NODE_COUNTERS] == [out["fp64"][1][k] for k in NODE_COUNTERS]
    pairs64 = out["fp64"][1]["direct_pair_evaluations"]
    assert abs(out["mixed"][1]["direct_pair_evaluations"] - pairs64) <= 1e-7 * pairs64
