"""Shared test setup: import paths, the `gpu` marker, and the CPU checkers (oracle)."""
from __future__ import annotations

import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "ap-cloud-cosmology_b200")
ORACLE = os.path.join(ROOT, "oracle")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)

REFERENCE_SRC = "/root/reference"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def _make(target: str) -> None:
    subprocess.run(["make", "-s", "-C", ORACLE, target], check=True)


@pytest.fixture(scope="session")
def oracle_lib():
    """The plain-C restatement, built on demand."""
    so = os.path.join(ORACLE, "liboracle.so")
    if not os.path.exists(so):
        _make("oracle")
    return so


@pytest.fixture(scope="session")
def reference_lib():
    """The reference's own code (oracle/_ref), built here when its sources are present;
    on a host without them the prebuilt library that travelled with the tree is used."""
    so = os.path.join(ORACLE, "_ref", "libapcref.so")
    if not os.path.exists(so):
        if not os.path.isdir(REFERENCE_SRC):
            pytest.skip("reference sources and prebuilt oracle/_ref both absent")
        _make("ref")
    return so


@pytest.fixture(scope="session")
def gpu_lib():
    """libapcloud_gpu.so; built here if missing (nvcc cross-compiles without a GPU)."""
    from apcloud import binding

    if not os.path.exists(binding.LIB_PATH):
        import importlib.util

        spec = importlib.util.spec_from_file_location("apc_build", os.path.join(PKG, "build.py"))
        mod = importlib.util.module_from_spec(spec)
        spec.loader.exec_module(mod)
        mod.build()
    return binding.LIB_PATH
