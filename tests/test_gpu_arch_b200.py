"""The compiled drop-in: the B200 specialisation of the reference's
ComputeUnitArchitecture (include/tdlb_compute_unit_arch_b200.hpp), built
against the reference's own headers into tests/cpp/_bin/arch_b200_main
(tests/cpp/Makefile; the binary travels with the tree), next to the
reference's CPU ComputeUnit in the same program. Both are driven through
ComputeUnitBase<float, 18, MemoryLayoutIJKL>* in main.cpp's order:
initialise, forcing with std::vector<PosPolar<long, float>>, the fixed
markers as excluded output points, then per step collision,
bounceBackBoundary, streamingPush, moments, forcing; at the end the B200
unit writes its vorticity slices through the reference's JPEG writer.

Tolerance (60^3 Rushton tank, 20 steps, relative L2 over the interior, as the
60^3 parity test): rho, u, F and Nu <= 1e-4; the Esotwist parity flag equal.
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "tests", "cpp", "_bin", "arch_b200_main")


def driver():
    if not os.path.exists(EXE):
        pytest.fail(f"{EXE} is not built (make -C tests/cpp, where the reference sources are)")
    return EXE


def gpu_present():
    try:
        import torch
        return torch.cuda.is_available()
    except ImportError:
        return False


def test_arch_b200_driver_fails_loudly_without_a_gpu(tmp_path):
    if gpu_present():
        pytest.skip("a GPU is present")
    r = subprocess.run([driver(), "Simple", "16", "2", str(tmp_path)], capture_output=True, text=True, timeout=120,
                       cwd=str(tmp_path))
    assert r.returncode == 3, r.stdout + r.stderr
    assert "no CUDA device" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
def test_arch_b200_specialisation_vs_reference_cpu_unit(gpu, tmp_path, streaming):
    r = subprocess.run([driver(), streaming, "60", "20", str(tmp_path)], capture_output=True, text=True,
                       timeout=600, cwd=str(tmp_path))
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    line = [ln for ln in r.stdout.splitlines() if ln.startswith("ok ")]
    assert line, r.stdout[-3000:]
    fields = dict(kv.split("=") for kv in line[-1].split()[1:])
    for key in ("rho", "u", "F", "Nu"):
        assert float(fields[key]) <= 1e-4, f"{key}: relative L2 {fields[key]}"
    assert fields["even"] == fields["even_ref"]
    assert int(fields["markers"]) > 1000
    assert fields["jpeg_xz"] == "1" and fields["jpeg_xy"] == "1"
