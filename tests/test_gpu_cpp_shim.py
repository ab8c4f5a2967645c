"""The C++20 host shim (chui-dev_b200/host/tree_pm_coordinator.hpp) drives the
library the way a CHUI host drives TreePmCoordinator: compiled here with g++,
run on the GPU, compared with the same solve through the Python binding, and
checked for the reference's exception type on an invalid cutoff."""
import os
import struct
import subprocess

import numpy as np
import pytest

import chui_treepm as ct
from chui_treepm import ics

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST = os.path.join(ROOT, "chui-dev_b200", "host")
BUILD = os.path.join(ROOT, "chui-dev_b200", "_build")


def test_cpp_shim_matches_python_binding(tmp_path):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    exe = tmp_path / "shim_example"
    subprocess.run(["g++", "-std=c++20", "-O2", os.path.join(HOST, "shim_example.cpp"), f"-L{BUILD}",
                    "-lchui_treepm", f"-Wl,-rpath,{BUILD}", "-o", str(exe)], check=True)
    # r_cut well inside half the box, so the production walk's subtree blocks apply
    x, y, z, *_ = ics.zeldovich_lattice(32, 40.0, 0.2, seed=21)
    n = len(x)
    m = np.full(n, 1.0 / n)
    box, mesh, theta, leaf, eps = 40.0, 32, 0.7, 16, 0.01
    fin = tmp_path / "in.bin"
    with open(fin, "wb") as f:
        f.write(struct.pack("<qdqdqd", n, box, mesh, theta, leaf, eps))
        for a in (x, y, z, m):
            f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    fout = tmp_path / "out.bin"
    subprocess.run([str(exe), str(fin), str(fout)], check=True)
    out = np.fromfile(fout, dtype=np.float64).reshape(6, n)
    # the shim asks for diagnostics, so its walk is the counted production walk
    cfg = ct.TreePmConfig(pm_grid_nx=mesh, pm_grid_ny=mesh, pm_grid_nz=mesh, box_x=box, box_y=box, box_z=box,
                          opening_theta=theta, max_leaf_size=leaf, softening=eps, diagnostics=2)
    with ct.TreePmCoordinator(cfg) as s:
        r = s.solve_active_set(x, y, z, m)
    ref = np.stack([r["ax"], r["ay"], r["az"]])
    scale = np.abs(ref).max()
    assert np.abs(out[:3] - ref).max() <= 1e-5 * scale
    # cadence reuse of the cached PM field gives the same force
    assert np.abs(out[3:] - out[:3]).max() <= 1e-5 * scale


def test_cosmosim_adapter_matches_reference(tmp_path):
    """The coordinator over the reference's own types, driven as the reference
    runtime drives TreePmCoordinator (chui-dev_b200/host/cosmosim_example.cpp,
    built by __graft_entry__.build() against the reference's headers), on the
    per-particle softening fixture: the reference's TreeSofteningView rules
    resolve the lanes, the forces meet the mixed bar against the reference's
    own solve, and a PM-reuse solve gives the same forces."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    exe = os.path.join(BUILD, "cosmosim_example")
    if not os.path.isfile(exe):
        pytest.skip("cosmosim_example not built (needs the reference's headers at build time)")
    from conftest import load_golden
    g = load_golden("softening_mixed")
    n = len(g["x"])
    asmth, rcut, theta, gconst, eps = (float(v) for v in g["params"])
    leaf, scheme, deconv, criterion, order = (int(v) for v in g["iparams"])
    fin = tmp_path / "in.bin"
    with open(fin, "wb") as f:
        f.write(struct.pack("<qdqdqdqq", n, float(g["box"][0]), int(g["mesh"][0]), theta, leaf, eps, deconv, 1))
        for a in (g["x"], g["y"], g["z"], g["m"], g["src_eps"], g["src_mask"].astype(np.float64)):
            f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    fout = tmp_path / "out.bin"
    subprocess.run([exe, str(fin), str(fout)], check=True)
    out = np.fromfile(fout, dtype=np.float64).reshape(6, n)
    ref = np.stack([g["ax"], g["ay"], g["az"]])
    den = np.linalg.norm(ref, axis=0)
    e = np.linalg.norm(out[:3] - ref, axis=0) / np.maximum(den, 1e-6 * np.median(den))
    assert np.median(e) <= 1e-4 and np.percentile(e, 99) <= 1e-3, (np.median(e), np.percentile(e, 99))
    assert np.abs(out[3:] - out[:3]).max() <= 1e-5 * np.abs(ref).max()
