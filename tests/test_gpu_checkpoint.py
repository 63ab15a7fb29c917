"""Checkpoint writer / reader in the reference's layout (ComputeUnit.hpp:318-439).

* The B200 writer's Q / F / Nu files match the reference writer's for the
  same run (interior; relative L2 within the step tolerance of the parity
  tests -- the two runs differ only by FP32 rounding), including the
  Esotwist writeMoments placement after an odd number of steps.
* The reference reads a B200 checkpoint and continues in step with the GPU;
  the GPU reads a reference checkpoint and continues in step with it.
* A B200 write -> read round trip continues bit-identically.
"""
import glob
import json
import os

import numpy as np
import pytest

from test_gpu_parity import random_markers, rel_l2, velocity

pytestmark = pytest.mark.gpu

ALPHA, BETA = 0.97, 1.9
DIMS = (9, 7, 11)
NU = 5e-4


def make_pair(tb, po, streaming, tmp, storage="fp32"):
    x, y, z = DIMS
    flow = po.Flow(initialRho=1.0, nu=NU, cs0=0.1, g3=0.8, alpha=ALPHA, beta=BETA, useLES=True)
    lat = po.CpuLattice("ref", x, y, z, flow, streaming, 4, tmpdir=str(tmp))
    cu = make_unit(tb, streaming, storage)
    return cu, lat


def make_unit(tb, streaming, storage="fp32"):
    x, y, z = DIMS
    return tb.ComputeUnit(x=x, y=y, z=z, nu=NU, cs0=0.1, g3=0.8, useLES=1, storage=storage, initialRho=1.0,
                          streaming=tb.STREAMING_SIMPLE if streaming == "Simple" else tb.STREAMING_ESOTWIST)


def marker_lists(tb, seed, count):
    x, y, z = DIMS
    rng = np.random.default_rng(seed)
    return [random_markers(tb, rng, x * z // 2, x, y, z, planes=[0, y // 2, y - 1]) for _ in range(count)]


def advance(units, lats, markers):
    for mk in markers:
        for lat in lats:
            lat.step(mk, ALPHA, BETA)
        for cu in units:
            cu.collision()
            cu.forcing(mk, ALPHA, BETA)


def start(units, lats, mk):
    for lat in lats:
        lat.initialise(1.0)
        lat.forcing(mk, ALPHA, BETA)
    for cu in units:
        cu.initialise(1.0)
        cu.forcing(mk, ALPHA, BETA)


def compare(cu, lat, nsteps, tag):
    """GPU against the reference CPU CU (no touched flags on that side)."""
    mg = cu.read_moments().astype(np.float64)
    mr = lat.get_moments()
    fg = cu.read_force().astype(np.float64)
    fr = lat.interior(lat.get_f())
    tol_u = 2e-6 * max(nsteps, 1)
    assert rel_l2(mg[..., 0], mr[..., 0]) <= tol_u, tag
    assert rel_l2(velocity(mg, fg), velocity(mr, fr)) <= tol_u, tag
    assert rel_l2(fg, fr) <= 5e-5, tag
    assert rel_l2(cu.read_nu(), lat.interior(lat.get_nu())) <= 5e-5, tag


def files(d):
    out = {}
    for p in glob.glob(os.path.join(d, "*")):
        out[os.path.basename(p)] = p
    return out


def interior(a, shape, width):
    x, y, z = shape
    return a.reshape(x + 2, y + 2, z + 2, width)[1:-1, 1:-1, 1:-1]


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
def test_b200_checkpoint_matches_reference_writer(gpu, ref_oracle, tmp_path, streaming):
    tb, po = gpu, ref_oracle
    cu, lat = make_pair(tb, po, streaming, tmp_path)
    mks = marker_lists(tb, 11, 4)
    start([cu], [lat], mks[0])
    advance([cu], [lat], mks[1:])          # 3 steps: Esotwist parity is odd
    dg = str(tmp_path / "b200")
    cu.checkpoint_write(dg, "device", {"RunningParams": {"step": 3, "angle": 0.0}})
    dr = lat.checkpoint_write("device", 3)
    fg, fr = files(dg), files(dr)
    assert sorted(fg) == sorted(fr)
    for name in fg:
        assert os.path.getsize(fg[name]) == os.path.getsize(fr[name]) or name.endswith(".json")
    qg = np.fromfile(fg["checkpoint_grid.0.0.0.device.Q"], np.float32)
    qr = np.fromfile(fr["checkpoint_grid.0.0.0.device.Q"], np.float32)
    qgi, qri = interior(qg, DIMS, 18), interior(qr, DIMS, 18)
    assert rel_l2(qgi[..., 0], qri[..., 0]) <= 1e-5          # density
    assert rel_l2(qgi[..., 1:4], qri[..., 1:4]) <= 2e-5      # momentum
    assert rel_l2(qgi, qri) <= 1e-4                          # all 18 moments
    ghost = np.ones((DIMS[0] + 2, DIMS[1] + 2, DIMS[2] + 2), bool)
    ghost[1:-1, 1:-1, 1:-1] = False
    assert not qg.reshape(ghost.shape + (18,))[ghost].any()
    Fg = np.fromfile(fg["checkpoint_grid.0.0.0.device.F"], np.float32)
    Fr = np.fromfile(fr["checkpoint_grid.0.0.0.device.F"], np.float32)
    assert rel_l2(interior(Fg, DIMS, 3), interior(Fr, DIMS, 3)) <= 5e-5
    assert np.array_equal(interior(Fg, DIMS, 3) != 0, interior(Fr, DIMS, 3) != 0)
    Ng = np.fromfile(fg["checkpoint_grid.0.0.0.device.Nu"], np.float32)
    Nr = np.fromfile(fr["checkpoint_grid.0.0.0.device.Nu"], np.float32)
    assert rel_l2(interior(Ng, DIMS, 1), interior(Nr, DIMS, 1)) <= 5e-5
    params = json.load(open(fg["AllParams.0.0.0.device.json"]))
    assert params["RunningParams"]["step"] == 3
    assert params["StreamingState"]["evenStep"] == lat.even_step
    assert params["ComputeUnitParams"]["x"] == DIMS[0]
    cu.close()


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
def test_reference_continues_from_b200_checkpoint(gpu, ref_oracle, tmp_path, streaming):
    tb, po = gpu, ref_oracle
    cu, lat = make_pair(tb, po, streaming, tmp_path)
    mks = marker_lists(tb, 12, 6)
    start([cu], [lat], mks[0])
    advance([cu], [lat], mks[1:4])
    dg = str(tmp_path / "b200")
    cu.checkpoint_write(dg, "device")
    back = po.CpuLattice("ref", *DIMS, lat.flow, streaming, 4, tmpdir=str(tmp_path))
    back.checkpoint_read(dg, "device")
    # the reference's reader drops evenStep; the B200 file carries it
    back.even_step = json.load(open(os.path.join(dg, "AllParams.0.0.0.device.json")))["StreamingState"]["evenStep"]
    advance([cu], [back], mks[4:])
    compare(cu, back, 5, "reference resumed from the B200 checkpoint")
    advance([], [lat], mks[4:])
    compare(cu, lat, 5, "uninterrupted reference")
    cu.close()


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
def test_b200_continues_from_reference_checkpoint(gpu, ref_oracle, tmp_path, streaming):
    tb, po = gpu, ref_oracle
    _, lat = make_pair(tb, po, streaming, tmp_path)
    mks = marker_lists(tb, 13, 5)
    start([], [lat], mks[0])
    advance([], [lat], mks[1:3])          # 2 steps: the parity is even again
    dr = lat.checkpoint_write("device", 2)
    cu = make_unit(tb, streaming)
    cu.checkpoint_read(dr, "device")
    assert cu.evenStep == lat.even_step
    advance([cu], [lat], mks[3:])
    compare(cu, lat, 2, "B200 resumed from the reference checkpoint")
    cu.close()


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
def test_round_trip_continues_bit_identically(gpu, tmp_path, streaming):
    tb = gpu
    a = make_unit(tb, streaming)
    mks = marker_lists(tb, 14, 7)
    start([a], [], mks[0])
    advance([a], [], mks[1:4])
    d = str(tmp_path / "rt")
    a.checkpoint_write(d, "device")
    b = make_unit(tb, streaming)
    b.checkpoint_read(d, "device")
    assert b.evenStep == a.evenStep
    advance([a, b], [], mks[4:])
    np.testing.assert_array_equal(a.read_moments(), b.read_moments())
    np.testing.assert_array_equal(a.read_force(), b.read_force())
    np.testing.assert_array_equal(a.read_nu(), b.read_nu())
    np.testing.assert_array_equal(a.read_touched(), b.read_touched())
    a.close()
    b.close()


def test_fp16_checkpoint_write_tracks_fp32(gpu, tmp_path):
    tb = gpu
    mks = marker_lists(tb, 15, 4)
    out = {}
    for storage in ("fp32", "fp16"):
        cu = make_unit(tb, "Simple", storage)
        start([cu], [], mks[0])
        advance([cu], [], mks[1:])
        d = str(tmp_path / storage)
        cu.checkpoint_write(d, "device")
        out[storage] = np.fromfile(os.path.join(d, "checkpoint_grid.0.0.0.device.Q"), np.float32)
        if storage == "fp16":
            with pytest.raises(tb.TdlbError, match="FP32"):
                cu.checkpoint_read(d, "device")
        cu.close()
    q32, q16 = interior(out["fp32"], DIMS, 18), interior(out["fp16"], DIMS, 18)
    assert rel_l2(q16[..., 0], q32[..., 0]) <= 2e-4
    assert rel_l2(q16[..., 1:4], q32[..., 1:4]) <= 2e-2


def test_checkpoint_read_errors(gpu, tmp_path):
    tb = gpu
    cu = make_unit(tb, "Simple")
    with pytest.raises(tb.TdlbError) as e:
        cu.checkpoint_read(str(tmp_path / "missing"), "device")
    assert e.value.code == -4
    cu.initialise(1.0)
    d = str(tmp_path / "ok")
    cu.checkpoint_write(d, "device")
    other = tb.ComputeUnit(x=DIMS[0] + 1, y=DIMS[1], z=DIMS[2], nu=NU)
    with pytest.raises(tb.TdlbError) as e:
        other.checkpoint_read(d, "device")
    assert e.value.code == -1
    os.truncate(os.path.join(d, "checkpoint_grid.0.0.0.device.Nu"), 16)
    with pytest.raises(tb.TdlbError) as e:
        cu.checkpoint_read(d, "device")
    assert e.value.code == -4
    cu.close()
    other.close()
