"""Resolution doubling on the device (doubleResolutionFullCU,
ComputeUnit.hpp:258-316; index map indexPreviousResolution :480-502).

The reference's own doubleResolutionFullCU is not run as the oracle: its
copy loop runs l < 19 over 18-entry records (:237), writing one float past
the end of its Q array. The test restates its index map instead: every new
cell holds the moments and Nu of old cell (i/2, j/2, k/2), F and the touched
flags are zero, checked bit for bit against the moments the old state read
back as. The doubled lattice then continues in step with the FP32
restatement started from the same state (handed over through the
checkpoint writer, which also places the Esotwist moments).
"""
import json
import os

import numpy as np
import pytest

from test_gpu_parity import compare, random_markers

pytestmark = pytest.mark.gpu

ALPHA, BETA = 0.97, 1.9


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
def test_double_resolution_copies_parent_cells_and_continues(gpu, port_oracle, tmp_path, streaming):
    tb, po = gpu, port_oracle
    x, y, z = 10, 8, 12
    rng = np.random.default_rng(5)
    cu = tb.ComputeUnit(x=x, y=y, z=z, nu=2e-3, cs0=0.1, g3=0.8, useLES=1, initialRho=1.0,
                        streaming=tb.STREAMING_SIMPLE if streaming == "Simple" else tb.STREAMING_ESOTWIST)
    cu.initialise(1.0)
    for _ in range(5):                       # 5 steps: the Esotwist parity is odd
        cu.collision()
        cu.forcing(random_markers(tb, rng, 40, x, y, z, planes=[1, 4, 6]), ALPHA, BETA)
    m_old = cu.read_moments()
    nu_old = cu.read_nu()
    even = cu.evenStep
    cu.doubleResolutionFullCU()
    assert (cu.x, cu.y, cu.z) == (2 * x, 2 * y, 2 * z)
    assert cu.evenStep == even
    m_new = cu.read_moments()
    ii, jj, kk = np.meshgrid(np.arange(2 * x) // 2, np.arange(2 * y) // 2, np.arange(2 * z) // 2, indexing="ij")
    np.testing.assert_array_equal(m_new, m_old[ii, jj, kk])
    np.testing.assert_array_equal(cu.read_nu(), nu_old[ii, jj, kk])
    assert not cu.read_force().any()
    assert not cu.read_touched().any()
    with pytest.raises(tb.TdlbError):
        cu.forcing_resident(ALPHA, BETA)     # the old markers are gone
    # continue at the new size against the restatement started from the same state
    d = str(tmp_path / "doubled")
    cu.checkpoint_write(d, "device")
    X, Y, Z = 2 * x, 2 * y, 2 * z
    lat = po.CpuLattice("port", X, Y, Z, po.Flow(initialRho=1.0, nu=2e-3, cs0=0.1, g3=0.8, useLES=True), streaming, 4)
    lat.set_q(np.fromfile(os.path.join(d, "checkpoint_grid.0.0.0.device.Q"), np.float32).astype(np.float64))
    lat.set_f(np.fromfile(os.path.join(d, "checkpoint_grid.0.0.0.device.F"), np.float32).astype(np.float64))
    lat.set_nu_field(np.fromfile(os.path.join(d, "checkpoint_grid.0.0.0.device.Nu"), np.float32).astype(np.float64))
    lat.even_step = json.load(open(os.path.join(d, "AllParams.0.0.0.device.json")))["StreamingState"]["evenStep"]
    for s in range(1, 4):
        mk = random_markers(tb, rng, 160, X, Y, Z, planes=[2, 8, 13])
        lat.step(mk, ALPHA, BETA)
        cu.collision()
        cu.forcing(mk, ALPHA, BETA)
        compare(cu, lat, s, f"step {s} after doubling")
    cu.close()


def test_double_resolution_rejections(gpu):
    tb = gpu
    cu = tb.ComputeUnit(x=8, y=8, z=8, nu=1e-3)
    with pytest.raises(tb.TdlbError):
        cu.doubleResolutionFullCU()          # not initialised
    cu.close()
    cu = tb.ComputeUnit(x=8, y=8, z=8, nu=1e-3, storage="fp16")
    cu.initialise(1.0)
    with pytest.raises(tb.TdlbError, match="FP32"):
        cu.doubleResolutionFullCU()
    cu.close()
