"""The reference's checkpoint format, pinned on the CPU by running the
reference's own checkpoint_write / checkpoint_read (ComputeUnit.hpp:318-439,
DiskOutputTree.h:560-589): the file names, the ghosted AoS sizes, that Q holds
exactly the CU's Q, and that the reference drops evenStep (the gap the B200
writer's "StreamingState" extension closes)."""
import glob
import json
import os

import numpy as np
import pytest

ALPHA, BETA = 0.97, 1.9


def _empty_markers():
    import tdlbcpp_b200 as tb
    return np.zeros(0, tb.MARKER_DTYPE)


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
def test_reference_checkpoint_layout(ref_oracle, tmp_path, streaming):
    po = ref_oracle
    x, y, z = 6, 5, 7
    flow = po.Flow(initialRho=1.0, nu=0.01, cs0=0.1, g3=0.8, alpha=ALPHA, beta=BETA, useLES=True)
    lat = po.CpuLattice("ref", x, y, z, flow, streaming, 4, tmpdir=str(tmp_path))
    lat.initialise(1.0)
    for _ in range(3):
        lat.step(_empty_markers(), ALPHA, BETA)
    d = lat.checkpoint_write("device", 3)
    assert d.endswith("_step_3")
    names = sorted(os.listdir(d))
    assert names == ["AllParams.0.0.0.device.json", "checkpoint_grid.0.0.0.device.F",
                     "checkpoint_grid.0.0.0.device.Nu", "checkpoint_grid.0.0.0.device.Q"]
    ng = (x + 2) * (y + 2) * (z + 2)
    assert os.path.getsize(os.path.join(d, "checkpoint_grid.0.0.0.device.Q")) == ng * 18 * 4
    assert os.path.getsize(os.path.join(d, "checkpoint_grid.0.0.0.device.F")) == ng * 3 * 4
    assert os.path.getsize(os.path.join(d, "checkpoint_grid.0.0.0.device.Nu")) == ng * 4
    q = np.fromfile(os.path.join(d, "checkpoint_grid.0.0.0.device.Q"), np.float32)
    np.testing.assert_array_equal(q, lat.get_q().astype(np.float32).ravel())
    params = json.load(open(glob.glob(os.path.join(d, "AllParams*.json"))[0]))
    for key in ("BinFileParams", "CheckpointParams", "ComputeUnitParams", "FlowParams", "GridParams",
                "OutputParams", "RunningParams"):
        assert key in params
    assert params["RunningParams"]["step"] == 3
    assert "StreamingState" not in params
    back = po.CpuLattice("ref", x, y, z, flow, streaming, 4, tmpdir=str(tmp_path))
    back.checkpoint_read(d, "device")
    np.testing.assert_array_equal(back.get_q(), lat.get_q())
    if streaming == "Esotwist":
        # three steps leave the parity odd; the reference's reader starts even
        assert lat.even_step is False and back.even_step is True


def test_reference_plane_dump_layout(ref_oracle, tmp_path):
    """savePlaneXZ<float, 4> (ComputeUnitOutput.hpp:354-447): 24-byte
    tDiskGrid<float, 4> records in (i, k) order with jGrid = j - 1 (ghosted j);
    no F records before any forcing."""
    import tdlbcpp_b200 as tb
    po = ref_oracle
    x, y, z = 5, 6, 7
    lat = po.CpuLattice("ref", x, y, z, po.Flow(initialRho=1.0, nu=0.01), "Simple", 4, tmpdir=str(tmp_path))
    lat.initialise(1.0)
    d = lat.save_plane_xz(3, 1)
    q = np.fromfile(os.path.join(d, "CUid.0.0.0.V5.QVec.bin"), tb.DISK_GRID4_DTYPE)
    f = np.fromfile(os.path.join(d, "CUid.0.0.0.V5.F3.bin"), tb.DISK_GRID3_DTYPE)
    assert len(q) == x * z and len(f) == 0
    ii, kk = np.meshgrid(np.arange(x), np.arange(z), indexing="ij")
    np.testing.assert_array_equal(q["iGrid"], ii.ravel())
    np.testing.assert_array_equal(q["kGrid"], kk.ravel())
    assert np.all(q["jGrid"] == 2)
    np.testing.assert_array_equal(q["q"][:, 0], 1.0)
    np.testing.assert_array_equal(q["q"][:, 1:], 0.0)
