"""Shared pytest setup: the `gpu` marker and paths to the package and oracle."""
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]
PKG = ROOT / "khrr-nbody_b200"
ORACLE = ROOT / "oracle"
GOLDEN = ROOT / "tests" / "golden"
for p in (PKG, ORACLE):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def libkhrr():
    """The in-tree libkhrr.so, built with its Makefile if it is missing."""
    import ctypes
    import subprocess
    so = PKG / "build" / "libkhrr.so"
    if not so.exists():
        r = subprocess.run(["make", "-C", str(PKG)], capture_output=True, text=True)
        assert r.returncode == 0, r.stdout + r.stderr
    return ctypes.CDLL(str(so))


@pytest.fixture(scope="session")
def oracle():
    from pyoracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    def load(name):
        return dict(np.load(GOLDEN / name))
    return load
