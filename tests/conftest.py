"""Shared fixtures.  `-m gpu` tests need a B200; everything else runs on CPU."""
from __future__ import annotations

import importlib.util
import json
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG_DIR = ROOT / "pbc-based-dmpf-monte-carlo-test_b200"
sys.path.insert(0, str(Path(__file__).resolve().parent))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100a)")


def load_package():
    """Import the product package (its directory name is not an identifier)."""
    if "cmc_b200" in sys.modules:
        return sys.modules["cmc_b200"]
    spec = importlib.util.spec_from_file_location("cmc_b200", PKG_DIR / "__init__.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["cmc_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def cmc():
    if not (PKG_DIR / "libcmc.so").exists():
        subprocess.run(["make", "-C", str(PKG_DIR), "-j4"], check=True, stdout=subprocess.DEVNULL)
    return load_package()


@pytest.fixture(scope="session")
def oracle():
    from oracle_binding import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def golden():
    return json.loads((ROOT / "tests/golden/golden.json").read_text())


@pytest.fixture(scope="session")
def ctx(cmc):
    c = cmc.Context(0)
    yield c
    c.close()
