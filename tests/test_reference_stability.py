"""Long-run behaviour of the reference's own CPU ComputeUnit on a small
Rushton tank (48^3, Re 1277, LES): with Simple streaming the reference's wall
rule at the lattice faces (keep the cell's own post-collision population,
Boundary.hpp / StreamingSimple.hpp) lets the flow blow up within a few
hundred steps, while the same tank with Esotwist streaming (periodic) stays
bounded. The B200 path reproduces the reference step for step, so its
Simple tanks do the same; this is why the batched and serving workloads run
Esotwist tanks.
"""
import numpy as np
import pytest

ALPHA, BETA = 0.97, 1.9


def run(po, tb, streaming, steps, check_every=50):
    edge = 48
    rt = tb.RushtonTurbine(edge, edge, edge, tip_speed=0.1, startup_steps=0)
    nu = tb.nu_from_reynolds(1276.9886727287553, 0.1, rt.blade_outer_radius())
    flow = po.Flow(initialRho=1.0, nu=nu, cs0=0.1, g3=0.8, alpha=ALPHA, beta=BETA, useLES=True)
    lat = po.CpuLattice("ref", edge, edge, edge, flow, streaming, 4)
    d1 = rt.increment(1)
    lat.initialise(1.0)
    lat.forcing(rt.forcing_list(d1, d1, nonupdating_delta=d1), ALPHA, BETA)
    angle, peak = d1, 0.0
    for s in range(2, steps + 2):
        d = rt.increment(s)
        angle += d
        lat.step(rt.forcing_list(angle, d, nonupdating_delta=d1), ALPHA, BETA)
        if s % check_every == 0:
            j = lat.get_moments()[..., 1:4]
            peak = float(np.nanmax(np.abs(j))) if np.isfinite(j).any() else float("inf")
            if not np.isfinite(j).all() or peak > 1.0:
                lat.close()
                return s, peak
    lat.close()
    return None, peak


@pytest.mark.parametrize("streaming,diverges", [("Simple", True), ("Esotwist", False)])
def test_reference_small_tank_long_run(ref_oracle, streaming, diverges):
    import tdlbcpp_b200 as tb
    step, peak = run(ref_oracle, tb, streaming, 400)
    if diverges:
        assert step is not None, f"reference Simple tank stayed bounded (max |j| {peak})"
    else:
        assert step is None and peak < 0.5, f"reference Esotwist tank grew to {peak} by step {step}"
