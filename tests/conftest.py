"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on
the CPU (the driver runs `pytest -m "not gpu"` on a machine without a GPU)."""
from __future__ import annotations

import importlib.util
import json
import os
import subprocess
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(REPO, "cuda-graph-traversal_b200")
GOLDEN = os.path.join(REPO, "tests", "golden")
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def load_package():
    """Imports cuda-graph-traversal_b200/ (a directory name that is not a
    Python identifier) as module `cgt_b200`, building libg500b.so first when
    it is missing and nvcc is available."""
    if "cgt_b200" in sys.modules:
        return sys.modules["cgt_b200"]
    lib = os.path.join(PKG_DIR, "lib", "libg500b.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-s", "-C", PKG_DIR, "-j8"], check=True)
    spec = importlib.util.spec_from_file_location("cgt_b200", os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["cgt_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


@pytest.fixture(scope="session")
def cgt():
    return load_package()


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


def load_golden(name: str):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def golden_host():
    return load_golden("ref_host_kat.json")


@pytest.fixture(scope="session", params=[12, 14])
def golden_dump(request):
    return load_golden(f"ref_s{request.param}.json")
