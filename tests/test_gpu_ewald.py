"""GPU TreePM forces against the direct FP64 Ewald sums stored in the fixtures.

The fixtures hold the reference's own Ewald summation
(tests/support/periodic_ewald_reference.cpp:202-400 in the reference; alpha =
2.5/L, real images +-3, reciprocal modes +-10, as
tests/validation/test_tree_pm_ewald_accuracy.cpp:695-706 sets them) at the first
few targets, next to the reference's TreePM forces. A TreePM force differs from
the Ewald force by the split truncation and the mesh (the reference's own
rel-L2 error is ~1e-2 for CIC without deconvolution, ~4e-4 for the clustered
CIC + deconvolution box). The GPU solve, in FP64 and in mixed precision, must
carry the reference's error and add next to nothing to it.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import chui_treepm as ct  # noqa: E402
from conftest import load_golden  # noqa: E402
from test_gpu_parity import cfg_for  # noqa: E402

pytestmark = pytest.mark.gpu

CASES = ["lattice16_cic", "config32", "clustered64k_cic"]


def _rel_l2(got, ref):
    return float(np.linalg.norm(got - ref) / np.linalg.norm(ref))


@pytest.fixture(scope="module")
def cuda_ok():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("mode", ["fp64", "mixed_production", "mixed_diagnostics"])
def test_error_against_ewald(cuda_ok, name, mode, record_property):
    g = load_golden(name)
    k = len(g["ewald_ax"])
    ewald = np.stack([g["ewald_ax"], g["ewald_ay"], g["ewald_az"]])
    ref = np.stack([g["ax"][:k], g["ay"][:k], g["az"][:k]])
    cfg = cfg_for(g, ct._abi.FP64 if mode == "fp64" else ct._abi.MIXED)
    cfg.diagnostics = 0 if mode == "mixed_production" else 1
    with ct.TreePmCoordinator(cfg) as s:
        r = s.solve_active_set(g["x"], g["y"], g["z"], g["m"])
    got = np.stack([r["ax"][:k], r["ay"][:k], r["az"][:k]])
    err_gpu = _rel_l2(got, ewald)
    err_ref = _rel_l2(ref, ewald)
    per_target = np.linalg.norm(got - ewald, axis=0) / np.linalg.norm(ewald, axis=0)
    record_property("rel_l2_vs_ewald", err_gpu)
    record_property("reference_rel_l2_vs_ewald", err_ref)
    record_property("median_rel_vs_ewald", float(np.median(per_target)))
    print(f"{name} {mode}: rel-L2 vs Ewald {err_gpu:.4e} (reference TreePM {err_ref:.4e}), "
          f"median per target {np.median(per_target):.3e}, max {per_target.max():.3e}")
    # the GPU solve carries the reference's truncation error and adds at most
    # 1e-5 of the Ewald force (FP64: round-off; mixed: FP32 pair arithmetic)
    assert abs(err_gpu - err_ref) <= 1e-5 + 1e-3 * err_ref, (err_gpu, err_ref)
    assert _rel_l2(got, ref) <= (1e-9 if mode == "fp64" else 1e-4), _rel_l2(got, ref)
