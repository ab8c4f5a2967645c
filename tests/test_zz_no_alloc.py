"""Allocation-free density entry point (chui_pm_assign_density_static) against
the allocating one (chui_pm_assign_density) on the same device inputs, called
through the C-ABI with ctypes.

The file name sorts last so the test also runs after every other GPU test in
the same process (the entry point's per-device set-up then happens late).
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from chui_treepm import _abi  # noqa: E402

pytestmark = pytest.mark.gpu

MESH = (32, 24, 40)
BOX = (10.0, 8.0, 12.0)


@pytest.fixture(scope="module")
def lib():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return _abi.load()


def make_config(lib, scheme, mesh=MESH):
    cfg = _abi.Config()
    assert lib.chui_treepm_config_default(C.byref(cfg)) == 0
    cfg.pm_grid_nx, cfg.pm_grid_ny, cfg.pm_grid_nz = mesh
    cfg.box_x, cfg.box_y, cfg.box_z = BOX
    cfg.assignment_scheme = scheme
    return cfg


def device_sources(n, seed, with_mass=True):
    rng = np.random.default_rng(seed)
    # includes coordinates outside [0, L): the deposit wraps them periodically
    pos = [torch.tensor(rng.uniform(-0.5 * L, 1.5 * L, n), dtype=torch.float64, device="cuda") for L in BOX]
    mass = torch.tensor(rng.uniform(0.5, 2.0, n), dtype=torch.float64, device="cuda") if with_mass else None
    src = _abi.Sources()
    src.count = n
    src.x, src.y, src.z = (p.data_ptr() for p in pos)
    src.mass = mass.data_ptr() if mass is not None else None
    src.uniform_mass = 0.0 if with_mass else 1.5
    return src, (pos, mass)


def last_error(lib):
    return lib.chui_treepm_last_error(None).decode()


@pytest.mark.parametrize("scheme", [_abi.CIC, _abi.TSC])
@pytest.mark.parametrize("with_mass", [True, False])
def test_static_density_matches_allocating_entry_point(lib, scheme, with_mass):
    cfg = make_config(lib, scheme)
    cells = MESH[0] * MESH[1] * MESH[2]
    src, keep = device_sources(40000, 11 + scheme, with_mass)

    handle = C.c_void_p()
    assert lib.chui_treepm_create(C.byref(cfg), C.byref(handle)) == 0
    try:
        ref = torch.empty(cells, dtype=torch.float64, device="cuda")
        assert lib.chui_pm_assign_density(handle, C.byref(src), C.c_void_p(ref.data_ptr()), _abi.DEVICE, None) == 0
        torch.cuda.synchronize()
        ref = ref.cpu().numpy()
    finally:
        lib.chui_treepm_destroy(handle)

    # two calls in a row: device output, then host output
    out_dev = torch.full((cells,), np.nan, dtype=torch.float64, device="cuda")
    rc = lib.chui_pm_assign_density_static(C.byref(cfg), C.byref(src), C.c_void_p(out_dev.data_ptr()),
                                           _abi.DEVICE, None)
    assert rc == 0, last_error(lib)
    out_host = np.full(cells, np.nan)
    rc = lib.chui_pm_assign_density_static(C.byref(cfg), C.byref(src), C.c_void_p(out_host.ctypes.data),
                                           _abi.HOST, None)
    assert rc == 0, last_error(lib)

    # FP64 atomics accumulate in a different order on every call
    tol = 1e-12 * np.abs(ref).max()
    assert np.abs(out_dev.cpu().numpy() - ref).max() <= tol
    assert np.abs(out_host - ref).max() <= tol
    cell_volume = BOX[0] * BOX[1] * BOX[2] / cells
    total = float(keep[1].sum()) if with_mass else 1.5 * 40000
    assert abs(out_host.sum() * cell_volume - total) <= 1e-10 * total


def test_static_density_rejects_what_it_cannot_serve(lib):
    src, keep = device_sources(1000, 5)
    out = torch.empty(_abi.STATIC_MAX_CELLS + 1, dtype=torch.float64, device="cuda")

    big = make_config(lib, _abi.CIC, mesh=(64, 64, 65))  # 266240 cells > 262144
    rc = lib.chui_pm_assign_density_static(C.byref(big), C.byref(src), C.c_void_p(out.data_ptr()), _abi.DEVICE, None)
    assert rc == _abi.ERANGE
    assert "exceeds the static scratch grid" in last_error(lib)

    cfg = make_config(lib, _abi.CIC)
    host_x = np.zeros(1000)
    host_src = _abi.Sources()
    host_src.count = 1000
    host_src.x = host_x.ctypes.data
    host_src.y = src.y
    host_src.z = src.z
    host_src.mass = src.mass
    rc = lib.chui_pm_assign_density_static(C.byref(cfg), C.byref(host_src), C.c_void_p(out.data_ptr()),
                                           _abi.DEVICE, None)
    assert rc == _abi.EINVAL
    assert "device memory" in last_error(lib)

    # the largest mesh the scratch grid holds still works after the rejections
    edge = make_config(lib, _abi.CIC, mesh=(64, 64, 64))
    rc = lib.chui_pm_assign_density_static(C.byref(edge), C.byref(src), C.c_void_p(out.data_ptr()), _abi.DEVICE, None)
    assert rc == 0, last_error(lib)
