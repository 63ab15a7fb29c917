"""Shared test set-up.

Markers:
  gpu  -- needs an sm_100 GPU and the built CUDA library; run with `-m gpu`.
          These tests fail (they do not skip) when the GPU path is missing,
          because the product has no CPU fallback.

The CPU oracles (oracle/libtdlb_oracle.so, oracle/_ref/libtdlb_ref.so) are
built on demand when missing and the sources are present.
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

REF_SRC = "/root/reference/tdlbcpp/src"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and the built CUDA library")


def _build(target: str):
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), target], check=True,
                   stdout=subprocess.DEVNULL, stderr=subprocess.PIPE)


@pytest.fixture(scope="session")
def port_oracle():
    from oracle import pyoracle as po
    if not po.available("port"):
        _build("port")
    return po


@pytest.fixture(scope="session")
def ref_oracle():
    from oracle import pyoracle as po
    if not po.available("ref"):
        if not os.path.isdir(REF_SRC):
            pytest.fail("oracle/_ref/libtdlb_ref.so is not built and the reference sources are absent")
        _build("ref")
    return po


@pytest.fixture(scope="session")
def tdlb():
    """The product package with its CUDA library loaded (no fallback)."""
    import tdlbcpp_b200 as tb
    tb.load_library()
    return tb


@pytest.fixture(scope="session")
def gpu(tdlb):
    """Asserts that a usable GPU is present: creates and destroys a lattice."""
    cu = tdlb.ComputeUnit(x=4, y=4, z=4, nu=1e-3)
    cu.close()
    return tdlb
