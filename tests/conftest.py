import glob
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")

from openpeec_b200.problem import Problem  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path")


def golden_names():
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def load_golden(name, sub=""):
    """(Problem, fixture dict) of a golden case written by tests/golden/make_golden.py
    (plane-wave cases live in the sub-directory "pw")."""
    z = dict(np.load(os.path.join(GOLDEN, sub, name + ".npz")))
    pz = {k[5:]: v for k, v in z.items() if k.startswith("prob_")}
    tmp = os.path.join(GOLDEN, ".__tmp_%d.npz" % os.getpid())
    np.savez(tmp, **pz)
    try:
        prob = Problem.load(tmp)
    finally:
        os.unlink(tmp)
    return prob, z


@pytest.fixture(scope="session")
def golden():
    cache = {}

    def get(name):
        if name not in cache:
            cache[name] = load_golden(name)
        return cache[name]
    return get


def relerr(a, b, floor=0.0):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor))) if a.size else 0.0
