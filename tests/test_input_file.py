"""The reference's own input file, as shipped, read by tdlb_create's parser.

main.cpp reads input_debug_gridx60_numSteps20.json (the reference's debug
input) with GridParams / FlowParams::getParamsFromJson (main.cpp:150-153)
and constructs its ComputeUnit from that FlowParams (main.cpp:242-256) before
calcNuAndRe_m (main.cpp:275) sets nu in main's own copy. The configuration
tdlb_create builds from the same text must equal, field by field, what the
reference's parsers give (oracle/_ref: tdlbref_read_input), nu included.

The file's values are also pinned here as SHIPPED_DEBUG_INPUT, which the GPU
test tests/test_gpu_parity.py::test_shipped_debug_input_vs_reference uses to
build the same unit on the box (the reference tree is not there).
"""
import os

import numpy as np
import pytest

SHIPPED_DEBUG_INPUT = {
    "x": 60, "y": 60, "z": 60, "multiStep": 1, "initialRho": 8.0, "nu": 0.0, "cs0": 0.12, "g3": 0.8,
    "alpha": 0.97, "beta": 1.9, "useLES": False, "streaming": "Esotwist",
}


def shipped_input_path(po):
    path = os.path.join(po.reference_root(), "input_debug_gridx60_numSteps20.json")
    if not os.path.exists(path):
        pytest.fail(f"the reference's input file {path} is missing")
    return path


def f32(v):
    return float(np.float32(v))


def test_shipped_input_file_matches_reference_parse(tdlb, ref_oracle):
    po = ref_oracle
    path = shipped_input_path(po)
    ref = po.ref_read_input(path)
    with open(path) as f:
        cfg = tdlb.config_from_json(f.read())
    assert (cfg.x, cfg.y, cfg.z) == (ref["x"], ref["y"], ref["z"])
    assert ref["multiStep"] == 1
    for key in ("initialRho", "nu", "cs0", "g3", "alpha", "beta"):
        assert getattr(cfg, key) == ref[key], key          # both float-rounded, bit for bit
    assert bool(cfg.useLES) == ref["useLES"]
    assert cfg.streaming == (tdlb.STREAMING_SIMPLE if ref["streaming"] == "Simple" else tdlb.STREAMING_ESOTWIST)
    assert cfg.storage == tdlb.STORAGE_FP32


def test_shipped_input_file_values_are_pinned(ref_oracle):
    """The constants the GPU test builds its unit from are the file's."""
    po = ref_oracle
    ref = po.ref_read_input(shipped_input_path(po))
    for key, val in SHIPPED_DEBUG_INPUT.items():
        want = f32(val) if isinstance(val, float) else val
        assert ref[key] == want, key
