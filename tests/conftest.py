"""Shared test set-up.

Markers:
  gpu  -- needs an sm_100 GPU and the built CUDA library; run with `-m gpu`.
          These tests fail (they do not skip) when the GPU path is missing,
          because the product has no CPU fallback.

The CPU oracles (oracle/libtdlb_oracle.so, oracle/_ref/libtdlb_ref.so) are
built on demand when missing (oracle/Makefile; the reference checkout is the
TDLB_REFERENCE environment variable, with the default the Makefile names).
"""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and the built CUDA library")


def _build(target: str):
    return subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), target],
                          stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)


@pytest.fixture(scope="session")
def port_oracle():
    from oracle import pyoracle as po
    if not po.available("port"):
        r = _build("port")
        if r.returncode:
            pytest.fail("building oracle/libtdlb_oracle.so failed:\n" + r.stdout[-2000:])
    return po


@pytest.fixture(scope="session")
def ref_oracle():
    from oracle import pyoracle as po
    if not po.available("ref"):
        r = _build("ref")
        if r.returncode:
            pytest.fail("oracle/_ref/libtdlb_ref.so is not built and building it failed "
                        "(are the reference sources present?):\n" + r.stdout[-2000:])
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
