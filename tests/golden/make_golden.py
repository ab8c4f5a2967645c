"""Generate the golden fixtures in tests/golden/ by running the reference's own
TreePM (oracle/_ref/treepm_ref, compiled from the reference's sources by
oracle/Makefile.ref) on seeded synthetic inputs.

    make -f oracle/Makefile.ref REF=<reference checkout> -j8
    python tests/golden/make_golden.py [name ...]   # all fixtures, or only the named ones

The reference has no stored golden vectors for this path; these fixtures are
its outputs on the same inputs, committed so the oracle and the CUDA path can
be checked without the reference present.
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "chui-dev_b200"))

import refio  # noqa: E402
from chui_treepm import ics  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

TREE_KEYS = ("ux", "uy", "uz", "anchors", "morton_key", "sorted_index", "center_x", "center_y",
             "center_z", "half", "mass", "com_x", "com_y", "com_z", "qxx", "qxy", "qxz", "qyy",
             "qyz", "qzz", "trace", "child_count", "child_index", "particle_begin", "particle_count")


ONLY = set(sys.argv[1:])


def save(name: str, p: refio.RefProblem, r, extra: dict | None = None, keep_tree=True):
    """r: the reference's result, or a callable producing it (run only for
    the selected fixtures)."""
    if ONLY and name not in ONLY:
        return
    if callable(r):
        r = r()
    d = {
        "x": p.x, "y": p.y, "z": p.z, "m": p.m,
        "vx": p.vx if p.vx is not None else np.zeros_like(p.x),
        "vy": p.vy if p.vy is not None else np.zeros_like(p.x),
        "vz": p.vz if p.vz is not None else np.zeros_like(p.x),
        "active": np.asarray(p.active if p.active is not None else [], dtype=np.uint32),
        "box": np.array(p.box), "mesh": np.array(p.mesh, dtype=np.int64),
        "params": np.array([p.asmth, p.rcut, p.theta, p.g, p.eps]),
        "iparams": np.array([p.leaf, p.scheme, p.deconv, p.criterion, p.order], dtype=np.int64),
        "kdk_factors": np.array([p.drift, p.kick1, p.kick2, p.drag1, p.drag2]),
        "counters": np.array([r["counters"][k] for k in ("visited", "accepted", "opened", "pairs",
                                                         "pruned", "pair_skips", "multipoles", "leaves")],
                             dtype=np.uint64),
    }
    for k in ("ax", "ay", "az", "pm_ax", "pm_ay", "pm_az", "tree_ax", "tree_ay", "tree_az", "nearest_r2"):
        d[k] = r[k]
    if keep_tree and r.get("n_nodes"):
        for k in TREE_KEYS:
            d[k] = r[k]
    if "density" in r:
        d["density"] = r["density"]
    for k in ("kdk_x", "kdk_y", "kdk_z", "kdk_vx", "kdk_vy", "kdk_vz", "kdk_ax", "kdk_ay", "kdk_az",
              "ewald_ax", "ewald_ay", "ewald_az"):
        if k in r:
            d[k] = r[k]
    if p.policy or p.prev_acc is not None:
        d["adaptive"] = np.array([p.policy, p.estimator, p.cutoff_policy], dtype=np.int64)
        d["adaptive_f"] = np.array([p.adaptive_angle, p.rel_tol, p.accel_floor])
        if p.prev_acc is not None:
            d["prev_acc"] = np.asarray(p.prev_acc, dtype=np.float64)
        if p.group_walk or p.gaussian_lookup:
            d["group"] = np.array([p.group_walk, p.gaussian_lookup], dtype=np.int64)
    if p.boundary:
        d["boundary"] = np.array([p.boundary], dtype=np.int64)
    if extra:
        d.update(extra)
    np.savez_compressed(os.path.join(OUT, name + ".npz"), **d)
    print(name, len(p.x), "nodes", r.get("n_nodes"), "counters", r["counters"])


def main():
    # 1. 16^3 Zel'dovich lattice, CIC, no deconvolution, unsoftened, one KDK step
    x, y, z, vx, vy, vz = ics.zeldovich_lattice(16, 10.0, 0.2, seed=11)
    m = np.full(len(x), 1.0 / len(x))
    p = refio.RefProblem(x, y, z, m, box=(10.0,) * 3, mesh=(16,) * 3, theta=0.5, leaf=16,
                         dump_density=1, kdk=1, drift=0.02, kick1=0.01, kick2=0.01,
                         vx=vx, vy=vy, vz=vz, ewald=32)
    save("lattice16_cic", p, lambda: refio.run(p))

    # 2. clustered: lattice + NFW halos, TSC + deconvolution, softened (accepted multipoles)
    x, y, z, vx, vy, vz = ics.zeldovich_lattice(20, 50.0, 0.3, seed=12)
    hx, hy, hz = ics.nfw_halos(3000, 6, 50.0, 2.0, seed=13, total_particles=len(x) + 3000)
    x, y, z = np.concatenate([x, hx]), np.concatenate([y, hy]), np.concatenate([z, hz])
    m = np.full(len(x), 2.0 / len(x))
    p = refio.RefProblem(x, y, z, m, box=(50.0,) * 3, mesh=(16,) * 3, theta=0.7, leaf=16, eps=0.05,
                         scheme=1, deconv=1, dump_density=1)
    save("clustered_tsc", p, lambda: refio.run(p))

    # 3. rectangular box, non-power-of-two mesh, non-canonical coordinates, active subset
    rng = np.random.default_rng(14)
    n = 3000
    box = (10.0, 8.0, 12.0)
    x = rng.uniform(-2.0, 12.0, n)
    y = rng.uniform(0.0, 8.0, n)
    z = rng.uniform(0.0, 12.0, n)
    x[:5] = [0.0, 10.0 - 1e-13, -1e-300, 5.0, 5.0]  # seam and coincident samples
    y[:5] = [0.0, 8.0 - 1e-12, 4.0, 4.0, 4.0]
    z[:5] = [0.0, 12.0 - 1e-12, 6.0, 6.0, 6.0]
    m = rng.uniform(0.5, 1.5, n) / n
    active = np.sort(rng.choice(n, 700, replace=False)).astype(np.uint32)
    active[:3] = [0, 3, 4]
    p = refio.RefProblem(x, y, z, m, box=box, mesh=(12, 10, 16), theta=0.5, leaf=8, eps=0.02, rcut=4.5,
                         active=active, dump_density=1)
    save("rect_active", p, lambda: refio.run(p))

    # 4. tiny cases: two-body, 24-particle quasi-uniform, duplicates deeper than a leaf
    p = refio.RefProblem(np.array([1.0, 1.7]), np.array([2.0, 2.1]), np.array([3.0, 2.6]),
                         np.array([1.0, 0.5]), box=(10.0,) * 3, mesh=(16,) * 3, theta=0.5, leaf=1)
    save("two_body", p, lambda: refio.run(p))
    rng = np.random.default_rng(15)
    x, y, z = (rng.uniform(0, 4.0, 24) for _ in range(3))
    p = refio.RefProblem(x, y, z, np.full(24, 1.0 / 24), box=(4.0,) * 3, mesh=(8,) * 3, theta=0.5,
                         leaf=4, eps=0.01, rcut=3.9)
    save("quasi24", p, lambda: refio.run(p))
    x = np.concatenate([np.full(20, 1.25), rng.uniform(0, 5.0, 200)])
    y = np.concatenate([np.full(20, 2.5), rng.uniform(0, 5.0, 200)])
    z = np.concatenate([np.full(20, 3.75), rng.uniform(0, 5.0, 200)])
    p = refio.RefProblem(x, y, z, np.full(220, 1.0 / 220), box=(5.0,) * 3, mesh=(8,) * 3, theta=0.5,
                         leaf=4, eps=0.02, rcut=3.9)
    save("duplicates", p, lambda: refio.run(p))

    # 5. the 32^3 configuration: L = 10 Mpc/h, lattice + Zel'dovich (P ~ k^-2, rms 0.2
    #    spacing), mesh 64^3, r_s = 1.25 cells, theta = 0.5, leaf 16, CIC, unsoftened,
    #    one KDK step, Ewald on 8 targets
    x, y, z, vx, vy, vz = ics.zeldovich_lattice(32, 10.0, 0.2, seed=1)
    m = np.full(len(x), 1.0 / len(x))
    p = refio.RefProblem(x, y, z, m, box=(10.0,) * 3, mesh=(64,) * 3, theta=0.5, leaf=16,
                         kdk=1, drift=0.02, kick1=0.01, kick2=0.01, vx=vx, vy=vy, vz=vz, ewald=8)
    save("config32", p, lambda: refio.run(p))

    # 6. adaptive relative policy (TreePmOptions::acceptance_policy = kAdaptiveRelative) on a
    #    clustered box: lattice + NFW halos, softened, leaf 8. The acceleration history is the
    #    reference's own strict-policy |a| on the same snapshot; a few entries are NaN (no
    #    history: COM-distance fallback), zero or below the floor (also the fallback).
    x, y, z, _, _, _ = ics.zeldovich_lattice(24, 20.0, 0.3, seed=21)
    hx, hy, hz = ics.nfw_halos(6000, 12, 20.0, 2.5, seed=22, total_particles=len(x) + 6000)
    x, y, z = np.concatenate([x, hx]), np.concatenate([y, hy]), np.concatenate([z, hz])
    m = np.full(len(x), 1.0 / len(x))
    common = dict(box=(20.0,) * 3, mesh=(32,) * 3, theta=0.5, leaf=8, eps=0.01, dump_tree=0)
    r0 = refio.run(refio.RefProblem(x, y, z, m, **common))
    prev = np.sqrt(r0["ax"] ** 2 + r0["ay"] ** 2 + r0["az"] ** 2)
    rng = np.random.default_rng(23)
    prev[rng.choice(len(x), 300, replace=False)] = np.nan
    prev[rng.choice(len(x), 40, replace=False)] = 0.0
    prev[rng.choice(len(x), 20, replace=False)] = 1e-31
    #    the production fast deck: relative monopole, COM-distance cutoff nodes,
    #    alpha 0.0025, maximum angle 1.0
    p = refio.RefProblem(x, y, z, m, **common, policy=1, estimator=1, cutoff_policy=1,
                         adaptive_angle=1.0, rel_tol=0.0025, prev_acc=prev)
    save("adaptive_monopole", p, lambda: refio.run(p))
    #    the default adaptive estimator: residual derivative, contain nodes, alpha 0.005,
    #    maximum angle 0.5; an active subset carries its own history slots
    active = np.sort(rng.choice(len(x), 5000, replace=False)).astype(np.uint32)
    p = refio.RefProblem(x, y, z, m, **common, policy=1, estimator=0, cutoff_policy=0,
                         adaptive_angle=0.5, rel_tol=0.005, prev_acc=prev[active], active=active)
    save("adaptive_residual", p, lambda: refio.run(p))
    #    the group walk (one conservative walk per leaf of targets, Gaussian Hermite pair
    #    table) on the fast deck, over all targets and over the active subset
    p = refio.RefProblem(x, y, z, m, **common, policy=1, estimator=1, cutoff_policy=1,
                         adaptive_angle=1.0, rel_tol=0.0025, prev_acc=prev, group_walk=1, gaussian_lookup=1)
    save("group_walk", p, lambda: refio.run(p))
    p = refio.RefProblem(x, y, z, m, **common, policy=1, estimator=1, cutoff_policy=0,
                         adaptive_angle=0.5, rel_tol=0.005, prev_acc=prev[active], active=active,
                         group_walk=1, gaussian_lookup=1)
    save("group_walk_active", p, lambda: refio.run(p))

    # 7. isolated/open boundaries (PmBoundaryCondition::kIsolatedOpen): a clustered
    #    distribution in the middle of the box plus particles on and beyond the faces
    #    (outside [0, L) they take no PM force and deposit nothing), zero-padded PM,
    #    non-periodic tree
    x, y, z, *_ = ics.clustered_box(12 ** 3, 10.0, 0.5, 6, 2.0, 0.4, 3)
    x, y, z = 2.5 + 0.5 * x, 2.5 + 0.5 * y, 2.5 + 0.5 * z
    x[:6] = [-0.1, 10.2, 3.0, 9.999, 0.0, 5.0]
    z[5] = 10.0
    rng = np.random.default_rng(31)
    m = rng.uniform(0.5, 1.5, len(x)) / len(x)
    p = refio.RefProblem(x, y, z, m, box=(10.0,) * 3, mesh=(16,) * 3, theta=0.5, leaf=8, boundary=1)
    save("isolated_cic", p, lambda: refio.run(p))
    active = np.sort(rng.choice(len(x), 600, replace=False)).astype(np.uint32)
    active[:4] = [0, 1, 3, 5]
    p = refio.RefProblem(x, y, z, m, box=(10.0,) * 3, mesh=(16,) * 3, theta=0.6, leaf=8, eps=0.02, scheme=1,
                         active=active, boundary=1)
    save("isolated_tsc_active", p, lambda: refio.run(p))

    # 8. the headline configuration's settings on a clustered periodic box of
    #    40^3 = 64000 particles at the 256^3 case's mean spacing (L = 31.25):
    #    50 % in 8 NFW halos over 3 decades, CIC with window deconvolution,
    #    theta 0.6, leaf 16, eps 0.001, mesh 40^3, r_s = 1.25 cells; Ewald
    #    sums at 16 targets
    x, y, z, *_ = ics.clustered_box(40 ** 3, 31.25, 0.5, 8, 3.0, 0.5, 81)
    m = np.full(len(x), 1.0 / len(x))
    p = refio.RefProblem(x, y, z, m, box=(31.25,) * 3, mesh=(40,) * 3, theta=0.6, leaf=16, eps=0.001,
                         scheme=0, deconv=1, dump_density=1, ewald=16)
    save("clustered64k_cic", p, lambda: refio.run(p))
    #    the large configuration's tree: theta 0.7, leaf 32, 60 % in 8 halos
    #    over 4 decades, same box, mesh and scheme
    x, y, z, *_ = ics.clustered_box(40 ** 3, 31.25, 0.6, 8, 4.0, 0.5, 82)
    m = np.full(len(x), 1.0 / len(x))
    p = refio.RefProblem(x, y, z, m, box=(31.25,) * 3, mesh=(40,) * 3, theta=0.7, leaf=32, eps=0.001,
                         scheme=0, deconv=1)
    save("clustered64k_t07_leaf32", p, lambda: refio.run(p))

    # 9. per-particle softening (TreeSofteningView): a clustered box whose halo
    #    particles take epsilon 0.02 and lattice particles 0.08 by override,
    #    with 5 % of the overrides off (the configured 0.05 applies); nodes
    #    mixing the two see the softening envelope guard. CIC + deconvolution,
    #    theta 0.7, leaf 16, quadrupoles (accepted multipoles).
    x, y, z, vx, vy, vz = ics.zeldovich_lattice(20, 50.0, 0.3, seed=91)
    hx, hy, hz = ics.nfw_halos(4000, 8, 50.0, 2.0, seed=92, total_particles=len(x) + 4000)
    n_lat = len(x)
    x, y, z = np.concatenate([x, hx]), np.concatenate([y, hy]), np.concatenate([z, hz])
    m = np.full(len(x), 2.0 / len(x))
    rng = np.random.default_rng(93)
    src_eps = np.where(np.arange(len(x)) < n_lat, 0.08, 0.02)
    src_mask = (rng.random(len(x)) >= 0.05).astype(np.uint8)
    common = dict(box=(50.0,) * 3, mesh=(16,) * 3, theta=0.7, leaf=16, eps=0.05, deconv=1)
    p = refio.RefProblem(x, y, z, m, **common, src_eps=src_eps, src_mask=src_mask)
    save("softening_mixed", p, lambda: refio.run(p), extra={"src_eps": src_eps, "src_mask": src_mask})
    #    an active subset with target sidecars: some targets override to 0.1 or
    #    0.0, the rest (mask 0) take the configured epsilon
    active = np.sort(rng.choice(len(x), 2500, replace=False)).astype(np.uint32)
    tgt_eps = rng.choice([0.1, 0.0, 0.03], len(active))
    tgt_mask = (rng.random(len(active)) >= 0.3).astype(np.uint8)
    p = refio.RefProblem(x, y, z, m, **common, active=active, src_eps=src_eps, src_mask=src_mask,
                         tgt_eps=tgt_eps, tgt_mask=tgt_mask, dump_tree=0)
    save("softening_active", p, lambda: refio.run(p), keep_tree=False,
         extra={"src_eps": src_eps, "src_mask": src_mask, "tgt_eps": tgt_eps, "tgt_mask": tgt_mask})


def kdk_factors():
    """The reference's CosmologicalTimeline::prepareStep factors for several
    backgrounds, scale factors and steps (flat LCDM, an open model with
    radiation, matter only), from the reference driver's --kdk-factors mode."""
    import subprocess
    if ONLY and "kdk_factors" not in ONLY:
        return
    cosmos = [(0.674, 0.315, 0.685, 0.0, 0.0), (0.7, 0.25, 0.7, 1e-4, 0.0499), (0.5, 1.0, 0.0, 0.0, 0.0)]
    steps = [(0.02, 1e-3), (0.1, 0.02), (0.5, 0.01), (1.0, 0.05), (0.9, 1e-6)]
    tspc = 3.0856775814913673e17  # seconds per code time unit (a kpc/(km/s) unit system)
    rows, out = [], []
    for c in cosmos:
        for a, dt in steps:
            r = subprocess.run([refio.binary(), "--kdk-factors", *(repr(v) for v in c), repr(tspc), repr(a), repr(dt)],
                               check=True, capture_output=True, text=True)
            rows.append(list(c) + [tspc, a, dt])
            out.append([float(v) for v in r.stdout.split()])
    np.savez_compressed(os.path.join(OUT, "kdk_factors.npz"), inputs=np.array(rows), factors=np.array(out))
    print("kdk_factors", len(rows))


if __name__ == "__main__":
    main()
    kdk_factors()
