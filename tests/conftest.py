"""Shared test setup.

Markers: ``gpu`` for tests that need a CUDA device (run on the B200 box);
everything else runs on CPU.  The libraries are built on demand (make is a
no-op when they are current)."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TESTS = os.path.join(ROOT, "tests")
for p in (ROOT, TESTS):
    if p not in sys.path:
        sys.path.insert(0, p)

REF_DIR = "/root/reference"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: longer CPU test")


def _ensure_built():
    if not os.path.exists(os.path.join(ROOT, "subgraphmatching_b200", "lib", "libsmx.so")):
        subprocess.run(["make", "-j8", "-C", "subgraphmatching_b200"], cwd=ROOT, check=True)
    if not os.path.exists(os.path.join(ROOT, "oracle", "lib", "libsmx_oracle.so")):
        subprocess.run(["make", "-C", "oracle", "port"], cwd=ROOT, check=True)


_ensure_built()


@pytest.fixture(scope="session")
def golden():
    with open(os.path.join(TESTS, "golden", "golden.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def port():
    from oracle import PortOracle

    return PortOracle()


@pytest.fixture(scope="session")
def ref():
    from oracle import RefOracle, available

    if not available()["ref"]:
        pytest.skip("reference oracle not built (needs the reference sources at build time)")
    return RefOracle()


@pytest.fixture(scope="session")
def emu():
    path = os.path.join(TESTS, "emu", "libsmx_emu.so")
    subprocess.run(["make", "-C", os.path.join(TESTS, "emu")], check=True, stdout=subprocess.DEVNULL)
    from emu_driver import Driver

    return Driver(path)


def has_gpu() -> bool:
    import subgraphmatching_b200 as smx

    return smx.device_count() > 0


@pytest.fixture(scope="session")
def gpu():
    if not has_gpu():
        pytest.skip("no CUDA device")
    return 0
