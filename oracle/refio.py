"""Test infrastructure (oracle): run the reference's own TreePM through
oracle/_ref/treepm_ref (built by oracle/Makefile.ref from the reference's
sources) and read its results back as numpy arrays.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline arm use this
module; the product never does.
"""
from __future__ import annotations

import os
import struct
import subprocess
import tempfile
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_BINARY = os.path.join(HERE, "_ref", "treepm_ref")          # x86-64-v3 (AVX2)
REF_BINARY_V4 = os.path.join(HERE, "_ref", "v4", "treepm_ref")  # x86-64-v4 (AVX-512)
_V4_FLAGS = ("avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl")


def _cpuinfo() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            return f.read()
    except OSError:
        return ""


def host_cpu() -> str:
    """The host CPU's model name (first processor entry)."""
    for line in _cpuinfo().splitlines():
        if line.startswith("model name"):
            return line.split(":", 1)[1].strip()
    return "unknown"


def binary() -> str:
    """The reference build for this host: the AVX-512 one where the CPU has
    AVX-512 and it was built, else the AVX2 one."""
    flags = set()
    for line in _cpuinfo().splitlines():
        if line.startswith("flags"):
            flags = set(line.split(":", 1)[1].split())
            break
    if all(f in flags for f in _V4_FLAGS) and os.access(REF_BINARY_V4, os.X_OK):
        return REF_BINARY_V4
    return REF_BINARY


def build_arch() -> str:
    return "x86-64-v4" if binary() == REF_BINARY_V4 else "x86-64-v3"


@dataclass
class RefProblem:
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    m: np.ndarray
    box: tuple = (1.0, 1.0, 1.0)
    mesh: tuple = (16, 16, 16)
    asmth: float = 1.25
    rcut: float = 6.25
    theta: float = 0.5
    g: float = 1.0
    eps: float = 0.0
    scale_factor: float = 1.0
    leaf: int = 16
    scheme: int = 0          # 0 CIC, 1 TSC
    deconv: int = 0
    criterion: int = 1       # 0 geometric, 1 com_distance, 2 relative
    order: int = 2           # 0 monopole, 2 quadrupole
    active: np.ndarray | None = None
    dump_tree: int = 1
    dump_density: int = 0
    kdk: int = 0
    repeats: int = 0
    ewald: int = 0
    drift: float = 0.0
    kick1: float = 0.0
    kick2: float = 0.0
    drag1: float = 1.0
    drag2: float = 1.0
    vx: np.ndarray | None = None
    vy: np.ndarray | None = None
    vz: np.ndarray | None = None
    # acceptance policy (TreePmOptions): 0 strict reference, 1 adaptive relative
    policy: int = 0
    estimator: int = 0       # adaptive: 0 residual derivative, 1 relative monopole
    cutoff_policy: int = 0   # adaptive: 0 contain node, 1 COM distance
    adaptive_angle: float = 0.25
    rel_tol: float = 0.005
    accel_floor: float = 1e-30
    prev_acc: np.ndarray | None = None  # per active target |a_previous|
    group_walk: int = 0       # TreePmOptions::group_walk_enabled
    gaussian_lookup: int = 0  # TreePmOptions::gaussian_pair_lookup_enabled
    boundary: int = 0         # PmBoundaryCondition: 0 periodic, 1 isolated/open
    # TreeSofteningView sidecars: source epsilon + override mask (per source),
    # target epsilon + override mask (per active slot)
    src_eps: np.ndarray | None = None
    src_mask: np.ndarray | None = None
    tgt_eps: np.ndarray | None = None
    tgt_mask: np.ndarray | None = None


def write_problem(path: str, p: RefProblem) -> None:
    n = len(p.x)
    zeros = np.zeros(n)
    active = np.asarray(p.active if p.active is not None else [], dtype=np.uint32)
    with open(path, "wb") as f:
        f.write(b"CHUIIN01")
        f.write(struct.pack("<q", n))
        f.write(struct.pack("<3d", *p.box))
        f.write(struct.pack("<3q", *p.mesh))
        f.write(struct.pack("<6d", p.asmth, p.rcut, p.theta, p.g, p.eps, p.scale_factor))
        f.write(struct.pack("<11q", p.leaf, p.scheme, p.deconv, p.criterion, p.order,
                            len(active), p.dump_tree, p.dump_density, p.kdk, p.repeats, p.ewald))
        f.write(struct.pack("<5d", p.drift, p.kick1, p.kick2, p.drag1, p.drag2))
        for a in (p.x, p.y, p.z, p.m,
                  p.vx if p.vx is not None else zeros,
                  p.vy if p.vy is not None else zeros,
                  p.vz if p.vz is not None else zeros):
            f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
        f.write(active.tobytes())
        grp = p.group_walk or p.gaussian_lookup or p.boundary
        if p.policy or p.prev_acc is not None or p.rel_tol != 0.005 or p.accel_floor != 1e-30 or grp:
            f.write(b"CHUIADP1")
            f.write(struct.pack("<4q", p.policy, p.estimator, p.cutoff_policy, int(p.prev_acc is not None)))
            f.write(struct.pack("<3d", p.adaptive_angle, p.rel_tol, p.accel_floor))
            if p.prev_acc is not None:
                prev = np.ascontiguousarray(p.prev_acc, dtype=np.float64)
                if len(prev) != (len(active) if len(active) else n):
                    raise ValueError("prev_acc needs one entry per active target")
                f.write(prev.tobytes())
            if grp:
                f.write(b"CHUIGRP1")
                f.write(struct.pack("<2q", p.group_walk, p.gaussian_lookup))
                if p.boundary:
                    f.write(b"CHUIISO1")
                    f.write(struct.pack("<q", p.boundary))
        if p.src_eps is not None or p.tgt_eps is not None:
            f.write(b"CHUISOF1")
            for eps, mask in ((p.src_eps, p.src_mask), (p.tgt_eps, p.tgt_mask)):
                e = np.ascontiguousarray(eps if eps is not None else [], dtype=np.float64)
                mk = np.ascontiguousarray(mask if mask is not None else np.ones(len(e)), dtype=np.uint8)
                f.write(struct.pack("<q", len(e)))
                f.write(e.tobytes())
                f.write(mk.tobytes())


class _Buf:
    def __init__(self, data: bytes):
        self.d = data
        self.o = 0

    def arr(self, dtype, count):
        a = np.frombuffer(self.d, dtype=dtype, count=count, offset=self.o).copy()
        self.o += a.nbytes
        return a

    def q(self):
        return int(self.arr(np.int64, 1)[0])


def read_result(path: str) -> dict:
    with open(path, "rb") as f:
        b = _Buf(f.read())
    assert b.d[:8] == b"CHUIOUT1"
    b.o = 8
    n = b.q()
    na = b.q()
    r: dict = {"n": n, "n_active": na}
    for k in ("ax", "ay", "az", "pm_ax", "pm_ay", "pm_az"):
        r[k] = b.arr(np.float64, na)
    for k in ("tree_ax", "tree_ay", "tree_az", "nearest_r2"):
        r[k] = b.arr(np.float64, n)
    r["first_ms"], r["pm_ms"], r["build_ms"], r["walk_ms"] = b.arr(np.float64, 4)
    reps = b.q()
    r["repeat_ms"] = b.arr(np.float64, reps)
    keys = ("visited", "accepted", "opened", "pairs", "pruned", "pair_skips", "multipoles", "leaves")
    r["counters"] = dict(zip(keys, (int(v) for v in b.arr(np.uint64, 8))))
    nn = b.q()
    r["n_nodes"] = nn
    if nn:
        for k in ("ux", "uy", "uz"):
            r[k] = b.arr(np.float64, n)
        r["anchors"] = b.arr(np.float64, 3)
        r["morton_key"] = b.arr(np.uint64, n)
        r["sorted_index"] = b.arr(np.uint32, n)
        for k in ("center_x", "center_y", "center_z", "half", "mass", "com_x", "com_y", "com_z",
                  "qxx", "qxy", "qxz", "qyy", "qyz", "qzz", "trace"):
            r[k] = b.arr(np.float64, nn)
        r["child_count"] = b.arr(np.uint32, nn)
        r["child_index"] = b.arr(np.uint32, 8 * nn)
        r["particle_begin"] = b.arr(np.uint32, nn)
        r["particle_count"] = b.arr(np.uint32, nn)
    cells = b.q()
    if cells:
        r["density"] = b.arr(np.float64, cells)
    kdk = b.q()
    if kdk:
        for k in ("kdk_x", "kdk_y", "kdk_z", "kdk_vx", "kdk_vy", "kdk_vz"):
            r[k] = b.arr(np.float64, n)
        for k in ("kdk_ax", "kdk_ay", "kdk_az"):
            r[k] = b.arr(np.float64, na)
    ew = b.q()
    if ew:
        nt = min(ew, na)
        for k in ("ewald_ax", "ewald_ay", "ewald_az"):
            r[k] = b.arr(np.float64, nt)
    if b.d[b.o:b.o + 8] == b"CHUIREP1":
        b.o += 8
        reps = b.q()
        # per repeat: PM, tree build and traversal milliseconds
        r["repeat_phases_ms"] = b.arr(np.float64, 3 * reps).reshape(reps, 3)
    return r


def available() -> bool:
    return os.path.isfile(REF_BINARY) and os.access(REF_BINARY, os.X_OK)


def run(p: RefProblem, threads: int | None = None, timeout: float | None = None) -> dict:
    """Run the reference TreePM on problem `p` and return its outputs."""
    if not available():
        raise FileNotFoundError(f"reference oracle binary missing: {REF_BINARY}")
    env = dict(os.environ)
    if threads is not None:
        env["OMP_NUM_THREADS"] = str(threads)
    with tempfile.TemporaryDirectory() as td:
        fin = os.path.join(td, "in.bin")
        fout = os.path.join(td, "out.bin")
        write_problem(fin, p)
        subprocess.run([binary(), fin, fout], check=True, env=env, timeout=timeout)
        return read_result(fout)
