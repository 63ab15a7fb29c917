"""bench.py's reference arm on the CPU: the reference's own step (the
compiled oracle/_ref library) timed on the host cores prints one JSON line
with the keys and meanings the main arm's line has, plus impl, cpu_baseline
and an e2e figure that moves no bytes between host and device."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


# Runs bench.py in this interpreter and, at exit, reports which of the
# project's shared libraries the process mapped (from /proc/self/maps).
_MAPS_WRAPPER = """
import atexit, runpy, sys
def _report():
    with open("/proc/self/maps") as f:
        maps = f.read()
    sys.stderr.write("MAPPED_B200=%d\\n" % ("libtdlb_b200.so" in maps))
    sys.stderr.write("MAPPED_REF=%d\\n" % ("libtdlb_ref.so" in maps))
atexit.register(_report)
sys.argv = ["bench.py"] + sys.argv[1:]
runpy.run_path("bench.py", run_name="__main__")
"""


def test_reference_arm_prints_one_contract_line(ref_oracle):
    out = subprocess.run([sys.executable, "-c", _MAPS_WRAPPER, "--impl", "reference", "--steps", "2",
                          "--warmup", "3"], cwd=ROOT, capture_output=True, text=True, timeout=600, check=True)
    lines = [ln for ln in out.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    # the reference arm runs the reference harness only: the B200 library is
    # never loaded into its process
    assert "MAPPED_REF=1" in out.stderr, out.stderr[-2000:]
    assert "MAPPED_B200=0" in out.stderr, out.stderr[-2000:]
    d = json.loads(lines[0])
    # it times exactly the steps and warm-up steps it was given
    assert d["steps"] == 2 and d["warmup"] == 3
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config"):
        assert key in d, key
    assert d["impl"] == "reference"
    assert d["metric"] == "MLUPS" and d["unit"] == "MLUPS" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] >= 1 and d["n_gpus"] == 1
    assert d["config"]["workload"].startswith("rushton-400^3")
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == d["value"] and cb["cores"] >= 1 and cb["sample"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_main_arm_fails_loudly_without_a_gpu():
    """No CPU fallback: without a GPU the measured arm exits non-zero and
    prints no JSON line."""
    import torch
    if torch.cuda.is_available():
        import pytest
        pytest.skip("a GPU is visible: the measured arm would run for real")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--steps", "3", "--warmup", "3",
                          "--no-cpu-baseline"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode != 0
    assert not [ln for ln in out.stdout.splitlines() if ln.strip().startswith("{")]
