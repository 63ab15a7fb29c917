"""tdlb_impeller_load_noalloc against tdlb_impeller_load (collected last).

The allocation-free entry point is for callers that cannot allocate device
memory once their run has started: a host application that gives the whole
GPU to its own memory pool up front, or a real-time loop that forbids
allocation after start-up. It writes the FP64 impeller load into a
caller-owned device buffer, using a fixed scratch array compiled into the
library instead of a cudaMalloc'd one.

Here, on a fresh handle, the first call is the allocation-free one (before
the allocating entry point has run on that handle), and it must give the
allocating entry point's answer on two calls in a row (with a time step in
between), within the tolerance the impeller-load parity test uses. Around
the second call the device's free memory must not change. Works alone in a
fresh process and after the other tests.
"""
import numpy as np
import pytest

ALPHA, BETA = 0.97, 1.9


def close_enough(got, want):
    # forces and torque: FP64 sums of the same FP32 terms in another order
    assert got[4] == want[4]
    scale = max(np.abs(want[:4]).max(), 1e-30)
    np.testing.assert_allclose(got[:4], want[:4], rtol=0, atol=2e-5 * scale)


@pytest.mark.gpu
def test_impeller_load_noalloc_matches_allocating_entry_point(gpu):
    import torch

    tb = gpu
    e = 40
    rt = tb.RushtonTurbine(e, e, e, tip_speed=0.1)
    d = rt.increment(1)
    nu = tb.nu_from_reynolds(7300.0, 0.1, rt.blade_outer_radius())
    cu = tb.ComputeUnit(x=e, y=e, z=e, nu=nu, cs0=0.1, useLES=1)
    cu.attach_rushton(rt, d, 0.0, d)
    cu.initialise(1.0)
    cu.forcing_resident(ALPHA, BETA)
    angle = 0.0
    for _ in range(2):
        angle += d
        cu.rotate_impeller(angle, d)
        cu.collision()
        cu.forcing_resident(ALPHA, BETA)

    # the caller's output buffer, allocated before the calls
    out = torch.full((5,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    for call in range(2):
        free_before = torch.cuda.mem_get_info()[0]
        cu.impeller_load_noalloc(out.data_ptr())      # on call 0: the handle's first load of any kind
        cu.synchronize()
        free_after = torch.cuda.mem_get_info()[0]
        got = out.cpu().numpy()
        if call == 1:
            # the first call may load the library's module onto the device
            # (lazy module loading, done by the driver); the second one
            # finds everything in place and allocates nothing
            assert free_after == free_before, f"free device memory changed by {free_before - free_after} bytes"
        want = cu.impeller_load()
        assert np.isfinite(got).all(), f"call {call}: {got}"
        close_enough(got, want)
        # advance one step so the second call sees different data
        angle += d
        cu.rotate_impeller(angle, d)
        cu.collision()
        cu.forcing_resident(ALPHA, BETA)
        out.fill_(float("nan"))
        torch.cuda.synchronize()
    cu.close()
