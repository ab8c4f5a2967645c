"""FP64 global momentum / energy checks on the device
(chui_treepm_momentum_energy) against numpy sums, momentum conservation of
the full TreePM force (net force ~ 0), and the host-memory kick and drift
against the device path."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import chui_treepm as ct  # noqa: E402
from chui_treepm import ics  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cuda_ok():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True


def test_momentum_energy_matches_numpy(cuda_ok):
    rng = np.random.default_rng(1)
    n = 100003
    m = rng.uniform(0.5, 2.0, n)
    v = [rng.normal(size=n) for _ in range(3)]
    a = [rng.normal(size=n) for _ in range(3)]
    cfg = ct.TreePmConfig(pm_grid_nx=16, pm_grid_ny=16, pm_grid_nz=16, box_x=10.0, box_y=10.0, box_z=10.0)
    with ct.TreePmCoordinator(cfg) as s:
        host = s.momentum_energy(m, *v, *a)
        dev = s.momentum_energy(*(torch.tensor(t, device="cuda") for t in (m, *v, *a)))
        uni = s.momentum_energy(None, *v, uniform_mass=1.5)
    for r in (host, dev):
        np.testing.assert_allclose(r["momentum"], [np.sum(m * vi) for vi in v], rtol=1e-12, atol=1e-9)
        np.testing.assert_allclose(r["net_force"], [np.sum(m * ai) for ai in a], rtol=1e-12, atol=1e-9)
        assert abs(r["kinetic_energy"] - 0.5 * np.sum(m * (v[0] ** 2 + v[1] ** 2 + v[2] ** 2))) <= 1e-12 * n
        assert abs(r["mass"] - m.sum()) <= 1e-12 * m.sum()
    assert abs(uni["mass"] - 1.5 * n) <= 1e-9 * n


@pytest.mark.parametrize("precision", [ct._abi.FP64, ct._abi.MIXED])
def test_total_force_conserves_momentum(cuda_ok, precision):
    x, y, z, *_ = ics.clustered_box(32 ** 3, 20.0, 0.4, 30, 2.0, 0.4, 3)
    m = np.full(len(x), 1.0 / len(x))
    cfg = ct.TreePmConfig(pm_grid_nx=32, pm_grid_ny=32, pm_grid_nz=32, box_x=20.0, box_y=20.0, box_z=20.0,
                          opening_theta=0.5, softening=0.01, precision=precision)
    with ct.TreePmCoordinator(cfg) as s:
        r = s.solve_active_set(x, y, z, m, short_range=True)
        tot = s.momentum_energy(m, r["ax"], r["ay"], r["az"], r["ax"], r["ay"], r["az"])
        tree = s.momentum_energy(m, r["tree_ax"], r["tree_ay"], r["tree_az"], r["tree_ax"], r["tree_ay"],
                                 r["tree_az"])
    scale = float(np.sum(m * np.sqrt(r["ax"] ** 2 + r["ay"] ** 2 + r["az"] ** 2)))
    tree_scale = float(np.sum(m * np.sqrt(r["tree_ax"] ** 2 + r["tree_ay"] ** 2 + r["tree_az"] ** 2)))
    # pair forces cancel pairwise up to rounding and the few strict multipoles
    assert np.abs(tree["net_force"]).max() <= 1e-5 * tree_scale
    assert np.abs(tot["net_force"]).max() <= 1e-3 * scale


@pytest.mark.parametrize("pinned", [True, False])
def test_host_kick_and_drift_match_device(cuda_ok, pinned):
    """Host-memory kick and drift run in chunks of 4 Mi elements on two
    streams; over several chunks and a ragged tail (pinned or pageable host
    arrays) they give the device path's results bit for bit, and the caller's
    stream sees the finished arrays."""
    n = (1 << 23) + 12345  # two whole chunks and a tail
    rng = np.random.default_rng(3)
    box = 10.0
    cfg = ct.TreePmConfig(pm_grid_nx=16, pm_grid_ny=16, pm_grid_nz=16, box_x=box, box_y=box, box_z=box)

    def host(a):
        if not pinned:
            return np.ascontiguousarray(a)
        return torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()

    p = [host(rng.random(n) * box) for _ in range(3)]
    v = [host(rng.standard_normal(n)) for _ in range(3)]
    a = [host(rng.standard_normal(n)) for _ in range(3)]
    dp = [torch.tensor(q, device="cuda") for q in p]
    dv = [torch.tensor(q, device="cuda") for q in v]
    da = [torch.tensor(q, device="cuda") for q in a]
    with ct.TreePmCoordinator(cfg) as s:
        s.kick(*v, *a, 0.3, 0.97)
        s.drift(*p, *v, 0.7)
        s.kick(*dv, *da, 0.3, 0.97)
        s.drift(*dp, *dv, 0.7)
        torch.cuda.synchronize()
    for h_arr, d_arr in zip(v + p, dv + dp):
        assert np.array_equal(h_arr, d_arr.cpu().numpy())
