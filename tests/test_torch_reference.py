"""Pins the FP64 torch formulation used as the reference gradient
(tests/treepm_torch_reference.py) against the C oracle's forces on small
periodic boxes where the strict walk accepts no multipole, so the oracle's
tree force is the direct sum inside r_cut."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

import oracle  # noqa: E402
import treepm_torch_reference as tr  # noqa: E402
from chui_treepm import ics  # noqa: E402


@pytest.mark.parametrize("scheme,deconv,eps", [(0, 1, 0.0), (1, 1, 0.05), (0, 0, 0.02)])
def test_torch_reference_matches_oracle_forces(scheme, deconv, eps):
    n_side, box = 8, 6.25
    mesh = (16, 16, 16)
    x, y, z, *_ = ics.zeldovich_lattice(n_side, box, 0.3, 5)
    m = np.full(len(x), 1.0 / len(x))
    p = oracle.make_params(box=(box,) * 3, mesh=mesh, theta=0.5, eps=eps, scheme=scheme, deconv=deconv)
    ref = oracle.treepm_solve(x, y, z, m, p)
    assert ref["counters"]["multipoles"] == 0
    prob = tr.Problem(mesh, (box,) * 3, eps=eps, scheme=scheme, deconv=bool(deconv))
    pos = [torch.tensor(v) for v in (x, y, z)]
    a = prob.accel(pos, torch.tensor(m))
    got = np.stack([t.numpy() for t in a])
    want = np.stack([ref["ax"], ref["ay"], ref["az"]])
    scale = np.abs(want).max()
    assert np.abs(got - want).max() <= 1e-10 * scale
