"""L2 prefetch of the step kernels (tdlb_set_l2_prefetch).

A full step launch has every eighth CTA issue bulk L2 prefetches of the
population spans the CTAs one wave further on will read. A prefetch moves
no data the kernel sees, so the stated tolerance is zero: velocity, density,
eddy viscosity, force and the impeller load are bit-identical with the
prefetch on and off, for both schemes, every storage form and every
cells-per-thread variant, on a lattice of several waves (96^3: 6912
one-cell tiles) and on one whose last rows end mid-tile (odd extents).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ALPHA, BETA = 0.97, 1.9


def run(tb, shape, streaming, storage, vec, prefetch, steps):
    x, y, z = shape
    rt = tb.RushtonTurbine(x, y, z, tip_speed=0.1, startup_steps=0)
    d = rt.increment(1)
    nu = tb.nu_from_reynolds(7300.0, 0.1, rt.blade_outer_radius())
    cu = tb.ComputeUnit(x=x, y=y, z=z, nu=nu, cs0=0.1, useLES=1, initialRho=1.0, storage=storage,
                        streaming=tb.STREAMING_SIMPLE if streaming == "Simple" else tb.STREAMING_ESOTWIST)
    cu.set_cells_per_thread(vec)
    cu.set_l2_prefetch(prefetch)
    cu.attach_rushton(rt, d, d, d)
    cu.initialise(1.0)
    cu.forcing_resident(ALPHA, BETA)
    angle = d
    for s in range(2, steps + 2):
        dd = rt.increment(s)
        angle += dd
        cu.rotate_impeller(angle, dd)
        cu.collision()
        cu.forcing_resident(ALPHA, BETA)
    rho, u = cu.read_velocity_density()
    out = {"rho": rho, "u": u, "nu": cu.read_nu(), "F": cu.read_force(), "load": np.array(cu.impeller_load())}
    cu.close()
    return out


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
@pytest.mark.parametrize("storage,vec", [("fp32", 1), ("fp32", 4), ("fp16", 2), ("fp16", 4), ("bf16", 1)])
@pytest.mark.parametrize("shape", [(96, 96, 96), (45, 38, 51)])
def test_prefetch_changes_no_result(gpu, streaming, storage, vec, shape):
    on = run(gpu, shape, streaming, storage, vec, True, 6)
    off = run(gpu, shape, streaming, storage, vec, False, 6)
    assert np.isfinite(on["u"]).all()
    for k in on:
        np.testing.assert_array_equal(on[k], off[k], err_msg=k)


def test_prefetch_switch_rejects_other_values(gpu):
    cu = gpu.ComputeUnit(x=8, y=8, z=8, nu=1e-3)
    try:
        assert cu.lib.tdlb_set_l2_prefetch(cu.h, 2) == -1   # TDLB_EINVAL
        cu.set_l2_prefetch(False)
        cu.set_l2_prefetch(True)
    finally:
        cu.close()
