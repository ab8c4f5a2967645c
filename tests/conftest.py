"""pytest configuration: the `gpu` marker and import paths.

Tests marked `gpu` need a CUDA device and the built extension; everything else
runs on CPU (the oracle against the reference's golden fixtures, host logic,
the C-ABI symbol table, and multi-process gloo tests).
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("chui-dev_b200", "oracle"):
    p = os.path.join(ROOT, sub)
    if p not in sys.path:
        sys.path.insert(0, p)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built extension")


def load_golden(name):
    import numpy as np
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def golden_params(g):
    """oracle.Params for a golden fixture."""
    import oracle
    asmth, rcut, theta, gconst, eps = (float(v) for v in g["params"])
    leaf, scheme, deconv, criterion, order = (int(v) for v in g["iparams"])
    adaptive = {}
    if "adaptive" in g:
        policy, estimator, cutoff_policy = (int(v) for v in g["adaptive"])
        angle, rel_tol, floor = (float(v) for v in g["adaptive_f"])
        adaptive = dict(policy=policy, estimator=estimator, cutoff_policy=cutoff_policy,
                        adaptive_angle=angle, rel_tol=rel_tol, accel_floor=floor)
    if "group" in g:
        adaptive["group_walk"], adaptive["gaussian_lookup"] = (int(v) for v in g["group"])
    if "boundary" in g:
        adaptive["boundary"] = int(g["boundary"][0])
    return oracle.make_params(box=tuple(g["box"]), mesh=tuple(int(v) for v in g["mesh"]), asmth=asmth,
                              rcut=rcut, theta=theta, g=gconst, eps=eps, leaf=leaf, scheme=scheme,
                              deconv=deconv, criterion=criterion, quadrupole=1 if order == 2 else 0,
                              **adaptive)


@pytest.fixture(scope="session")
def golden():
    return load_golden
