"""Shared pytest setup.

* marker ``gpu``: needs a CUDA device (B200); everything else runs on CPU.
* ``qvti`` fixture: the product's Python binding (q-vti_b200/qvti.py, ctypes
  over libqvti.so); ``oracle`` fixture: the FP64 CPU oracle (test checker).
"""
import glob
import importlib.util
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TESTS = os.path.join(ROOT, "tests")
GOLDEN = os.path.join(TESTS, "golden")
sys.path.insert(0, TESTS)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: test needs a CUDA GPU (B200)")


def load_qvti():
    spec = importlib.util.spec_from_file_location("qvti_b200", os.path.join(ROOT, "q-vti_b200", "qvti.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def qvti():
    return load_qvti()


@pytest.fixture(scope="session")
def oracle():
    import oracle as o
    return o


def load_golden(name):
    g = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    c = {}
    for k, v in g.items():
        if v.ndim == 0 and k not in ("velp", "vels", "rho", "gama_p", "gama_s"):
            c[k] = v.item()
        else:
            c[k] = v
    shape = (int(c["ntx"]), int(c["nty"]), int(c["ntz"]))
    for k in ("velp", "vels", "rho", "gama_p", "gama_s"):
        if np.ndim(c[k]) == 0:
            c[k] = np.full(shape, c[k], np.float32)
    return c


def golden_names():
    return sorted(os.path.splitext(os.path.basename(p))[0] for p in glob.glob(os.path.join(GOLDEN, "*.npz")))


def snap_keys(c):
    return sorted(int(k.split("_")[1]) for k in c if k.startswith("snap_"))
