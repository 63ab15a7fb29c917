"""The C++ ComputeUnit mirror (include/tdlb_compute_unit_b200.hpp) driven by
a main.cpp-shaped program (tests/cpp/drop_in_main.cpp) through the C ABI."""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build_driver(tmp_path):
    exe = str(tmp_path / "drop_in")
    lib_dir = os.path.join(ROOT, "tdlbcpp_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "drop_in_main.cpp"), "-L" + lib_dir, "-ltdlb_b200",
                    "-Wl,-rpath," + lib_dir, "-o", exe], check=True)
    return exe


def input_json(edge=30, streaming="Simple"):
    return json.dumps({
        "GridParams": {"x": edge, "y": edge, "z": edge, "multiStep": 1},
        "FlowParams": {"initialRho": 1.0, "reMNonDimensional": 7300.0, "uav": 0.1, "cs0": 0.1, "g3": 0.8,
                       "nu": 0.0, "alpha": 0.97, "beta": 1.9, "useLES": True, "streaming": streaming},
    })


def gpu_present():
    try:
        import torch
        return torch.cuda.is_available()
    except ImportError:
        return False


def test_cpp_driver_fails_loudly_without_gpu(tdlb, tmp_path):
    if gpu_present():
        pytest.skip("a GPU is present")
    exe = build_driver(tmp_path)
    r = subprocess.run([exe, input_json()], capture_output=True, text=True)
    assert r.returncode == 3
    assert "no CUDA device" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
def test_cpp_driver_runs_a_tank(gpu, tmp_path, streaming):
    exe = build_driver(tmp_path)
    r = subprocess.run([exe, input_json(30, streaming)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    fields = dict(kv.split("=") for kv in r.stdout.split()[1:])
    assert int(fields["cells"]) == 30 ** 3
    assert abs(float(fields["mass"]) / 30 ** 3 - 1.0) < 1e-3
    assert float(fields["absmom"]) > 0
