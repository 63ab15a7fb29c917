"""tdlb_impeller_load_async: the load of the last forcing pass queued with its
copy on the unit's stream, for callers that prepare the next step on the host
meanwhile (bench.py's end-to-end loop). Same reduction as
tdlb_impeller_load, so the stated tolerance is zero: bit-identical, into
pinned host memory and into device memory, and the blades uploaded for the
next step after the call do not change the queued result."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ALPHA, BETA = 0.97, 1.9


def test_async_load_equals_blocking_load(gpu):
    import torch
    tb = gpu
    e = 40
    rt = tb.RushtonTurbine(e, e, e, tip_speed=0.1, startup_steps=0)
    d = rt.increment(1)
    cu = tb.ComputeUnit(x=e, y=e, z=e, nu=1e-3, cs0=0.1, useLES=1)
    cu.attach_rushton(rt, d, d, d)
    cu.initialise(1.0)
    cu.forcing_resident(ALPHA, BETA)
    angle = d
    pinned = torch.empty(5, dtype=torch.float64, pin_memory=True)
    dev = torch.empty(5, dtype=torch.float64, device="cuda")
    for s in range(2, 6):
        angle += rt.increment(s)
        cu.set_rotating_markers(rt.rotating(angle, rt.increment(s)))
        cu.collision()
        cu.forcing_resident(ALPHA, BETA)
        want = cu.impeller_load()
        pinned.fill_(np.nan)
        cu.impeller_load_async(pinned.data_ptr())
        cu.impeller_load_async(dev.data_ptr())
        # the next step's blades, queued after the loads
        cu.set_rotating_markers(rt.rotating(angle + 0.3, rt.increment(s)))
        cu.synchronize()
        np.testing.assert_array_equal(pinned.numpy(), want)
        np.testing.assert_array_equal(dev.cpu().numpy(), want)
        cu.set_rotating_markers(rt.rotating(angle, rt.increment(s)))
    cu.close()
