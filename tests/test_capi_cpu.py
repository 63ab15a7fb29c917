"""CPU-side checks of the C ABI: the library loads and exports every
declared entry point, host-only logic (input JSON, geometry, the IBM
scheduler) behaves, and the GPU path fails loudly where there is no GPU."""
import ctypes
import json
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in sorted(os.listdir(os.path.join(ROOT, "include"))) if f.endswith(".h")]


def declared_symbols():
    names = set()
    for path in HEADERS:
        text = open(path).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(tdlb_\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol(tdlb):
    lib = ctypes.CDLL(tdlb.library_path())
    syms = declared_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def input_json(**overrides):
    """A reference-style input file (input_debug_gridx60_numSteps20.json keys)."""
    d = {
        "GridParams": {"ngx": 1, "ngy": 1, "ngz": 1, "x": 60, "y": 60, "z": 60, "multiStep": 1,
                       "strMinQVecPrecision": "float"},
        "FlowParams": {"initialRho": 1.0, "reMNonDimensional": 7300.0, "uav": 0.1, "cs0": 0.1, "g3": 0.8,
                       "nu": 0.0, "fx0": 0.0, "fy0": 0.0, "fz0": 0.0, "Re_m": 0.0, "Re_f": 0.0, "uf": 0.0,
                       "alpha": 0.97, "beta": 1.9, "useLES": True, "collision": "EgglesSomers",
                       "streaming": "Simple"},
        "RunningParams": {"step": 1, "angle": 0.0, "num_steps": 20, "impellerStartupStepsUntilNormalSpeed": 30,
                          "numStepsForAverageCalc": 10, "repeatPrintTimerToFile": 20, "repeatPrintTimerToStdOut": 10,
                          "runningDataFileDir": ".", "runningDataFilePrefix": "debug",
                          "runningDataFileAppendTime": True, "doubleResolutionAtStep": 0},
    }
    for sec, kv in overrides.items():
        d[sec].update(kv)
    return json.dumps(d)


def create_rc(tdlb, text):
    h = ctypes.c_void_p()
    rc = tdlb.load_library().tdlb_create(text.encode(), 0, ctypes.byref(h))
    msg = tdlb.load_library().tdlb_last_error(None).decode()
    if rc == 0:
        tdlb.load_library().tdlb_destroy(h)
    return rc, msg


def test_malformed_json_is_rejected(tdlb):
    rc, msg = create_rc(tdlb, "{ not json")
    assert rc == -6 and "input JSON" in msg


def test_missing_key_is_rejected(tdlb):
    d = json.loads(input_json())
    del d["FlowParams"]["cs0"]
    rc, msg = create_rc(tdlb, json.dumps(d))
    assert rc == -6 and "cs0" in msg


def test_ghost_width_other_than_one_is_rejected(tdlb):
    rc, msg = create_rc(tdlb, input_json(GridParams={"multiStep": 2}))
    assert rc == -1 and "multiStep" in msg


def test_no_gpu_means_an_error_not_a_fallback(tdlb):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    rc, msg = create_rc(tdlb, input_json())
    assert rc == -2, msg
    with pytest.raises(tdlb.TdlbError):
        tdlb.ComputeUnit(x=8, y=8, z=8)


def test_nu_from_reynolds_matches_calcNuAndRe_m(tdlb):
    # FlowParams.hpp:65-70 with T=float: Re_m = Re*pi/2, nu = uav*R/Re_m
    re_m = np.float32(7300.0 * np.pi / 2.0)
    want = np.float32(np.float32(0.1) * np.float32(10) / re_m)
    assert tdlb.nu_from_reynolds(7300.0, 0.1, 10) == float(want)


@pytest.mark.parametrize("edge", [32, 60, 96])
def test_rushton_geometry_in_range_and_classes(tdlb, edge):
    rt = tdlb.RushtonTurbine(edge, edge, edge, tip_speed=0.1, startup_steps=50)
    fixed, nonupd, rot = rt.fixed(), rt.rotating_nonupdating(rt.increment(1)), rt.rotating(0.7, rt.increment(1))
    for m in (fixed, nonupd, rot):
        assert len(m) > 0
        assert (m["i"] >= 0).all() and (m["i"] < edge).all()
        assert (m["j"] >= 0).all() and (m["j"] < edge).all()
        assert (m["k"] >= 0).all() and (m["k"] < edge).all()
        assert (np.abs(m["iCartFraction"]) <= 0.5).all() and (np.abs(m["kCartFraction"]) <= 0.5).all()
        # wall inset keeps every stencil off the periodic seam
        assert (m["i"] >= 1).all() and (m["i"] <= edge - 2).all()
    assert (fixed["uDelta"] == 0).all() and (fixed["wDelta"] == 0).all()
    assert rt.blade_outer_radius() == int(edge / 6)
    # blade tip speed = tip_speed at normal speed
    full = rt.increment(10 ** 6)
    tip = rt.rotating(0.0, full)
    speed = np.hypot(tip["uDelta"], tip["wDelta"]).max()
    assert abs(speed - 0.1) < 0.02
    assert rt.increment(25) == pytest.approx(full * 0.5)


# SHA-256 prefixes of the generated marker lists (fixed, rotating-non-updating,
# rotating at angle 0.7): the oracle and the GPU take the same list, and the
# list order sets the level schedule, so a faster generator must give these
# bytes exactly.
GEOMETRY_PINS = {
    (48, 48, 48): (7392, 443, 150, "76d4ffcc758a2111", "a2c76de5feec425a", "29c4b35af3ec1c5f"),
    (61, 50, 47): (10150, 554, 180, "9be4de741eb34b70", "659e487721025ada", "7d4d155a98f65973"),
}


@pytest.mark.parametrize("dims", sorted(GEOMETRY_PINS))
def test_rushton_geometry_bytes_pinned(tdlb, dims):
    import hashlib
    rt = tdlb.RushtonTurbine(*dims, tip_speed=0.1, startup_steps=0)
    lists = (rt.fixed(), rt.rotating_nonupdating(rt.increment(1)), rt.rotating(0.7, rt.increment(1)))
    pin = GEOMETRY_PINS[dims]
    assert tuple(len(m) for m in lists) == pin[:3]
    assert tuple(hashlib.sha256(m.tobytes()).hexdigest()[:16] for m in lists) == pin[3:]


def _stencil(m, x, z):
    cells = []
    for k1 in (-1, 0, 1):
        for i1 in (-1, 0, 1):
            cells.append((((m["i"] + i1) % x) * z + (m["k"] + k1) % z))
    return cells


def check_schedule(markers, lev, x, z):
    """Same-level markers of a plane share no cell; markers sharing a cell
    are on increasing levels in list order."""
    last = {}
    for q, m in enumerate(markers):
        for c in _stencil(m, x, z):
            key = (int(m["j"]), int(c))
            if key in last:
                prev = last[key]
                assert lev[prev] < lev[q], (prev, q)
            last[key] = q


def test_scheduler_invariants_random(tdlb):
    rng = np.random.default_rng(7)
    x, y, z = 12, 5, 9
    m = np.zeros(400, tdlb.MARKER_DTYPE)
    m["i"] = rng.integers(0, x, 400)
    m["j"] = rng.integers(0, y, 400)
    m["k"] = rng.integers(0, z, 400)
    lev, mx = tdlb.schedule_levels(m, x, y, z)
    check_schedule(m, lev, x, z)
    assert mx == lev.max() + 1


def test_scheduler_invariants_rushton(tdlb):
    e = 40
    rt = tdlb.RushtonTurbine(e, e, e, tip_speed=0.1)
    m = rt.forcing_list(0.3, rt.increment(1))
    lev, mx = tdlb.schedule_levels(m, e, e, e)
    check_schedule(m, lev, e, e)
    assert mx <= 24   # the generator's ordering keeps the level walk short


def test_scheduler_rejects_out_of_range(tdlb):
    m = np.zeros(1, tdlb.MARKER_DTYPE)
    m["i"] = 5
    with pytest.raises(tdlb.TdlbError):
        tdlb.schedule_levels(m, 5, 5, 5)
