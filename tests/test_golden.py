"""The committed golden fixtures pin the oracles on the CPU.

tests/golden/rushton16_6steps.npz was made by tests/golden/make_golden.py
from the reference's own CPU ComputeUnit (oracle/_ref, compiled in place):
a seeded 16^3 Rushton tank, 6 steps, FP32, Simple and Esotwist. Running the
same sequence again, the reference reproduces the fixture bit for bit, and
so does the C restatement in FP32 (it keeps the reference's operand types
and order). The GPU parity test against the same fixture is in
test_gpu_parity.py."""
import importlib.util
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "rushton16_6steps.npz")


def generator():
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(ROOT, "tests", "golden", "make_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
@pytest.mark.parametrize("kind", ["ref", "port"])
def test_oracles_reproduce_the_golden_fixture(port_oracle, ref_oracle, kind, streaming):
    g = np.load(GOLDEN)
    gen = generator()
    assert int(g["edge"]) == gen.EDGE and int(g["steps"]) == gen.STEPS
    got = gen.run(kind, streaming)
    for key in ("rho", "u", "F", "Nu"):
        want = g[f"{streaming}_{key}"]
        assert want.shape == got[key].shape, key
        assert np.isfinite(want).all(), key
        np.testing.assert_array_equal(got[key], want, err_msg=f"{kind} {streaming} {key}")
