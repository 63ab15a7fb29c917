"""Generates the golden fixtures of tests/golden/ from the reference itself.

The reference's own CPU ComputeUnit (oracle/_ref/libtdlb_ref.so, compiled in
place from the reference sources by oracle/Makefile) runs a seeded 16^3
Rushton tank for 6 steps in FP32, Simple and Esotwist streaming, with the
main-loop order of main.cpp:305 and :336-455 (forcing once, then per step:
impeller increment, collision, streaming, moments, forcing) and the
project's own marker generator (the same list the GPU path takes). The
fixture holds density, velocity u = (j + F/2)/rho, F and Nu of the interior
cells, FP32, (i, j, k) order.

Run from the repository root after `make -C oracle ref`:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import pyoracle as po  # noqa: E402  (test infrastructure: the checker)
import tdlbcpp_b200 as tb          # noqa: E402  (host-only geometry; no GPU needed)

EDGE, STEPS = 16, 6
RE, TIP, STARTUP = 7300.0, 0.1, 30
ALPHA, BETA = 0.97, 1.9
OUT = os.path.join(ROOT, "tests", "golden", "rushton16_6steps.npz")


def run(kind, streaming, edge=EDGE, steps=STEPS):
    """The reference main-loop sequence on a CPU lattice; returns the fields."""
    nu = tb.nu_from_reynolds(RE, TIP, edge // 6)
    rt = tb.RushtonTurbine(edge, edge, edge, tip_speed=TIP, startup_steps=STARTUP)
    flow = po.Flow(initialRho=1.0, nu=nu, cs0=0.1, g3=0.8, useLES=True)
    lat = po.CpuLattice(kind, edge, edge, edge, flow, streaming, 4)
    angle = 0.0
    d0 = rt.increment(1)
    fixed, nonupd = rt.fixed(), rt.rotating_nonupdating(d0)
    lat.initialise(1.0)
    lat.forcing(np.concatenate([fixed, nonupd, rt.rotating(angle, d0)]), ALPHA, BETA)
    for step in range(2, steps + 2):
        d = rt.increment(step)
        angle += d
        lat.step(np.concatenate([fixed, nonupd, rt.rotating(angle, d)]), ALPHA, BETA)
    m = lat.get_moments()
    f = lat.interior(lat.get_f())
    nu_field = lat.interior(lat.get_nu())
    lat.close()
    rho = m[..., 0]
    u = (m[..., 1:4] + 0.5 * f) / rho[..., None]
    return {"rho": rho.astype(np.float32), "u": u.astype(np.float32), "F": f.astype(np.float32),
            "Nu": nu_field.astype(np.float32)}


def main():
    out = {"edge": np.int32(EDGE), "steps": np.int32(STEPS)}
    for streaming in ("Simple", "Esotwist"):
        for key, v in run("ref", streaming).items():
            out[f"{streaming}_{key}"] = v
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
