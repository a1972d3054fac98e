"""Shared test set-up: import paths, the `gpu` marker, fixture loading."""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "pseudotransientstokes.jl_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on a B200)")


def pytest_sessionstart(session):
    """Bring libptstokes.so and the oracle up to date (no-op when already built)."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("pts_build", os.path.join(PKG, "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.build(quiet=True)
    import oracle

    oracle.build()


def load_golden(name):
    """A reference fixture (tests/golden/<name>.json): metadata, P array, X vector."""
    with open(os.path.join(GOLDEN, name + ".json")) as fh:
        d = json.load(fh)
    P = np.array([float.fromhex(h) for h in d["P"]["hex"]]).reshape(d["P"]["size"], order="F")
    X = np.array([float.fromhex(h) for h in d["X"]["hex"]])
    return d, P, X


def julia_isapprox(a, b):
    """Julia's default `isapprox` on arrays: norm(a-b) <= sqrt(eps)*max(norm(a), norm(b))."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return np.linalg.norm(a - b) <= np.sqrt(np.finfo(np.float64).eps) * max(np.linalg.norm(a), np.linalg.norm(b))


@pytest.fixture(scope="session")
def gpu_lib():
    """libptstokes.so, on a machine with a CUDA GPU."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import ptstokes
    return ptstokes.load()
