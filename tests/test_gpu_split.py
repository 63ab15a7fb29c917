"""Split steps: the outer chunks of a step run on the handle's stream while
the previous forcing pass and the inner chunks (marker stencils and, for
Esotwist, their neighbours) run on a second stream.

Every cell computes what the single launch computes, so the stated tolerance
is zero: velocity, density, eddy viscosity, force, touched flags and the FP64
impeller load are bit-identical with overlap on and off. The zone must hold
every cell a forcing pass touches (and, for Esotwist, every periodic
neighbour of one), at every impeller angle the run visits.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ALPHA, BETA = 0.97, 1.9


def run(tb, edge, streaming, storage, overlap, steps, host_blades=False, check_zone=None):
    rt = tb.RushtonTurbine(edge, edge, edge, tip_speed=0.1, startup_steps=0)
    d = rt.increment(1)
    nu = tb.nu_from_reynolds(7300.0, 0.1, rt.blade_outer_radius())
    cu = tb.ComputeUnit(x=edge, y=edge, z=edge, nu=nu, cs0=0.1, useLES=1, initialRho=1.0, storage=storage,
                        streaming=tb.STREAMING_SIMPLE if streaming == "Simple" else tb.STREAMING_ESOTWIST)
    cu.set_overlap("always" if overlap else False)
    cu.attach_rushton(rt, d, d, d)
    if storage != "fp32":
        cu.set_residual_box(0, 0, 0, 0, 0, 0)   # a step with a residual box never splits
        cu.set_cells_per_thread(1)              # nor one with several cells per thread
    cu.initialise(1.0)
    cu.forcing_resident(ALPHA, BETA)
    angle = d
    loads = []
    for s in range(2, steps + 2):
        dd = rt.increment(s)
        angle += dd
        if host_blades:
            cu.set_rotating_markers(rt.rotating(angle, dd))
        else:
            cu.rotate_impeller(angle, dd)
        cu.collision()
        cu.forcing_resident(ALPHA, BETA)
        if check_zone is not None and s % 7 == 0:
            check_zone(cu)
        if s % 5 == 0:                # most steps run with no join in between
            loads.append(cu.impeller_load())
    rho, u = cu.read_velocity_density()
    out = {"rho": rho, "u": u, "nu": cu.read_nu(), "F": cu.read_force(), "touched": cu.read_touched(),
           "loads": np.array(loads)}
    cu.close()
    return out


def zone_checker(streaming):
    def check(cu):
        zone = cu.read_zone().astype(bool)
        touched = cu.read_touched().astype(bool)
        assert touched.any()
        assert not (touched & ~zone).any(), "a touched cell lies outside the split-step zone"
        if streaming == "Esotwist":
            for di in (-1, 0, 1):
                for dj in (-1, 0, 1):
                    for dk in (-1, 0, 1):
                        nb = np.roll(touched, (di, dj, dk), axis=(0, 1, 2))
                        assert not (nb & ~zone).any(), "an Esotwist neighbour of a stencil cell is outside the zone"
    return check


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
@pytest.mark.parametrize("storage", ["fp32", "fp16"])
def test_split_step_is_bit_identical(gpu, streaming, storage):
    tb = gpu
    a = run(tb, 48, streaming, storage, True, 24, check_zone=zone_checker(streaming))
    b = run(tb, 48, streaming, storage, False, 24)
    for key in a:
        np.testing.assert_array_equal(a[key], b[key], err_msg=key)


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
def test_split_step_with_host_blades(gpu, streaming):
    """Blades uploaded by the host each step (the end-to-end path) are checked
    against the zone before the next split step."""
    tb = gpu
    a = run(tb, 40, streaming, "fp32", True, 12, host_blades=True, check_zone=zone_checker(streaming))
    b = run(tb, 40, streaming, "fp32", False, 12, host_blades=True)
    for key in a:
        np.testing.assert_array_equal(a[key], b[key], err_msg=key)


def test_split_step_launch_accounting(gpu):
    tb = gpu
    e = 40
    rt = tb.RushtonTurbine(e, e, e, tip_speed=0.1, startup_steps=0)
    d = rt.increment(1)
    cu = tb.ComputeUnit(x=e, y=e, z=e, nu=1e-3, cs0=0.1, useLES=1, streaming=tb.STREAMING_ESOTWIST)
    cu.set_overlap("always")
    cu.attach_rushton(rt, d, d, d)
    cu.initialise(1.0)
    cu.forcing_resident(ALPHA, BETA)
    cu.collision()                    # from moments: one launch
    cu.forcing_resident(ALPHA, BETA)
    zone = cu.read_zone()
    assert 0.0 < zone.mean() <= 1.0
    cu.set_kernel_timing(True)
    n0 = cu.kernel_launches()
    for s in range(3):
        cu.rotate_impeller(d * (s + 2), d)
        cu.collision()
        cu.forcing_resident(ALPHA, BETA)
    cu.join()
    ms, n = cu.kernel_time()
    assert n == 3 * (2 if zone.mean() < 1.0 else 1) and ms > 0.0   # outer + inner per split step
    assert cu.kernel_launches() - n0 >= 3 * (1 + 2 + 2)
    cu.set_cells_per_thread(4)        # split steps need one cell per thread
    with pytest.raises(tb.TdlbError):
        cu.read_zone()
    cu.set_cells_per_thread(1)
    cu.set_overlap(True)              # mode 1: this small tank is mostly stencil cells
    if zone.mean() > 0.6:
        with pytest.raises(tb.TdlbError):
            cu.read_zone()
    cu.set_overlap(False)
    with pytest.raises(tb.TdlbError):
        cu.read_zone()
    cu.close()


def test_zone_of_a_large_tank_is_small(gpu):
    """At 192^3 the stencil chunks (Esotwist, with neighbours) are a minority,
    so mode 1 splits; the default mode does not."""
    tb = gpu
    e = 192
    rt = tb.RushtonTurbine(e, e, e, tip_speed=0.1, startup_steps=0)
    d = rt.increment(1)
    cu = tb.ComputeUnit(x=e, y=e, z=e, nu=1e-3, cs0=0.1, useLES=1, streaming=tb.STREAMING_ESOTWIST)
    cu.attach_rushton(rt, d, d, d)
    with pytest.raises(tb.TdlbError):
        cu.read_zone()
    cu.set_overlap(True)
    cu.initialise(1.0)
    frac = cu.read_zone().mean()
    assert 0.0 < frac <= 0.6
    cu.close()
