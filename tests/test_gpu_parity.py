"""GPU parity tests: the CUDA path (through the C ABI) against the CPU oracle.

Integer work is compared bit for bit:
  * transport (streaming with an identity collision) on integer-coded
    populations, Simple wall rule and Esotwist index maps;
  * the immersed-boundary touched-cell flags (the reference's O field);
  * marker positions (host list == what the device applied).
Floating-point fields are compared by relative L2 norm against the
reference's FP32 arithmetic (the restatement, pinned bit-identical to the
reference compiled in place):
  * density and velocity:            rel. L2 <= 2e-6 per step, capped 2e-5
  * IBM force F and eddy viscosity:  rel. L2 <= 5e-5
The GPU computes in FP32 with fused multiply-adds and a factored moment
transform, so it rounds differently from the CPU; the bounds cover that
rounding with margin, not algorithmic differences (which would be O(1e-2)).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ALPHA, BETA = 0.97, 1.9


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0)


def coded_state(x, y, z):
    """Distinct exactly-representable codes: (cell * 18 + slot)."""
    n = x * y * z
    assert n * 18 < 2 ** 24
    return (np.arange(n * 18, dtype=np.float64).reshape(x, y, z, 18) + 1.0)


def ghosted(interior, fill=-7.0):
    x, y, z, q = interior.shape
    g = np.full((x + 2, y + 2, z + 2, q), fill)
    g[1:-1, 1:-1, 1:-1] = interior
    return g


# ---------------------------------------------------------------- transport

@pytest.mark.parametrize("vec", [1, 2, 4])
@pytest.mark.parametrize("dims", [(3, 3, 3), (4, 5, 6), (7, 3, 5), (5, 6, 37), (2, 9, 70), (1, 1, 1), (3, 2, 131)])
def test_transport_simple_bit_exact(gpu, port_oracle, dims, vec):
    tb, po = gpu, port_oracle
    x, y, z = dims
    codes = coded_state(x, y, z)
    cu = tb.ComputeUnit(x=x, y=y, z=z, nu=1e-3)
    cu.set_cells_per_thread(vec)
    cu.debug_set_state(codes, holds_moments=False)
    ref = po.CpuLattice("port", x, y, z, po.Flow(), "Simple", 8)
    ref.set_q(ghosted(codes))
    for _ in range(3):
        cu.debug_transport()
        ref.transport()
        np.testing.assert_array_equal(cu.debug_get_state().astype(np.float64), ref.get_q()[1:-1, 1:-1, 1:-1])
    cu.close()


@pytest.mark.parametrize("vec", [1, 2, 4])
@pytest.mark.parametrize("dims", [(3, 3, 3), (4, 5, 6), (7, 3, 5), (5, 6, 37), (2, 9, 70), (1, 2, 1), (3, 2, 131)])
def test_transport_esotwist_bit_exact(gpu, port_oracle, dims, vec):
    tb, po = gpu, port_oracle
    x, y, z = dims
    codes = coded_state(x, y, z)
    cu = tb.ComputeUnit(x=x, y=y, z=z, nu=1e-3, streaming=tb.STREAMING_ESOTWIST)
    cu.set_cells_per_thread(vec)
    cu.debug_set_state(codes, holds_moments=False)
    ref = po.CpuLattice("port", x, y, z, po.Flow(), "Esotwist", 8)
    ref.set_q(ghosted(codes))
    ref.even_step = True
    for _ in range(4):
        cu.debug_transport()
        ref.transport()
        assert cu.evenStep == ref.even_step
        np.testing.assert_array_equal(cu.debug_get_state().astype(np.float64), ref.get_q()[1:-1, 1:-1, 1:-1])
    cu.close()


def test_esotwist_transport_matches_reference_maps(gpu, ref_oracle):
    """Directly against the reference's AccessField code on its own coding."""
    tb, po = gpu, ref_oracle
    x, y, z = 4, 5, 6
    coded = po.coded_fill(x, y, z).astype(np.float64)
    for nsteps in (1, 2, 3):
        cu = tb.ComputeUnit(x=x, y=y, z=z, nu=1e-3, streaming=tb.STREAMING_ESOTWIST)
        cu.debug_set_state(coded[1:-1, 1:-1, 1:-1], holds_moments=False)
        for _ in range(nsteps):
            cu.debug_transport()
        want = po.kat_esotwist("ref", x, y, z, True, nsteps, False)[1:-1, 1:-1, 1:-1]
        np.testing.assert_array_equal(cu.debug_get_state().astype(np.uint64), want)
        cu.close()


def test_simple_transport_matches_reference_push(gpu, ref_oracle):
    tb, po = gpu, ref_oracle
    for dims in [(3, 3, 3), (4, 5, 6)]:
        x, y, z = dims
        coded = po.coded_fill(x, y, z).astype(np.float64)
        cu = tb.ComputeUnit(x=x, y=y, z=z, nu=1e-3)
        cu.debug_set_state(coded[1:-1, 1:-1, 1:-1], holds_moments=False)
        cu.debug_transport()
        want = po.kat_simple_stream("ref", True, x, y, z)[1:-1, 1:-1, 1:-1]
        np.testing.assert_array_equal(cu.debug_get_state().astype(np.uint64), want)
        cu.close()
    # and the reference's committed golden vectors (3x3x3 push)
    golden = po.kat_simple_golden(True)[1:-1, 1:-1, 1:-1]
    coded = po.coded_fill(3, 3, 3).astype(np.float64)
    cu = tb.ComputeUnit(x=3, y=3, z=3, nu=1e-3)
    cu.debug_set_state(coded[1:-1, 1:-1, 1:-1], holds_moments=False)
    cu.debug_transport()
    np.testing.assert_array_equal(cu.debug_get_state().astype(np.uint64), golden)
    cu.close()


# ---------------------------------------------------------------- physics

def random_markers(tb, rng, n, x, y, z, planes=None):
    m = np.zeros(n, tb.MARKER_DTYPE)
    m["i"] = rng.integers(0, x, n)
    m["j"] = rng.integers(0, y, n) if planes is None else rng.choice(planes, n)
    m["k"] = rng.integers(0, z, n)
    m["iCartFraction"] = rng.uniform(-0.5, 0.5, n)
    m["kCartFraction"] = rng.uniform(-0.5, 0.5, n)
    m["uDelta"] = rng.uniform(-0.05, 0.05, n)
    m["vDelta"] = rng.uniform(-0.05, 0.05, n)
    m["wDelta"] = rng.uniform(-0.05, 0.05, n)
    return m


def velocity(m, f):
    """QVec.hpp:385-394 in double from moments and F."""
    rho = m[..., 0]
    return (m[..., 1:4] + 0.5 * f) / rho[..., None]


def compare(cu, lat, nsteps, tag):
    mg = cu.read_moments().astype(np.float64)
    mr = lat.get_moments()
    fg = cu.read_force().astype(np.float64)
    fr = lat.interior(lat.get_f())
    tol_u = min(2e-5, 2e-6 * max(nsteps, 1))
    e_rho = rel_l2(mg[..., 0], mr[..., 0])
    e_u = rel_l2(velocity(mg, fg), velocity(mr, fr))
    e_f = rel_l2(fg, fr)
    assert e_rho <= tol_u, f"{tag}: rho rel L2 {e_rho:.3e}"
    assert e_u <= tol_u, f"{tag}: u rel L2 {e_u:.3e}"
    assert e_f <= 5e-5, f"{tag}: F rel L2 {e_f:.3e}"
    if lat.flow.useLES:
        e_nu = rel_l2(cu.read_nu(), lat.interior(lat.get_nu()))
        assert e_nu <= 5e-5, f"{tag}: Nu rel L2 {e_nu:.3e}"
    np.testing.assert_array_equal(cu.read_touched(), lat.interior(lat.get_o()), err_msg=f"{tag}: touched flags")
    return e_rho, e_u, e_f


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
@pytest.mark.parametrize("les", [True, False])
# (2, 5, 6) and (7, 4, 2): a marker's 3 x 3 stencil wraps onto itself in x or
# z, so its updates must stay sequential (the in-place path for distinct
# cells is not taken)
@pytest.mark.parametrize("dims", [(5, 5, 5), (9, 7, 11), (12, 10, 40), (2, 5, 6), (7, 4, 2)])
def test_step_parity_random_markers(gpu, port_oracle, streaming, les, dims):
    tb, po = gpu, port_oracle
    x, y, z = dims
    rng = np.random.default_rng(x * 100 + y * 10 + z + les)
    nu = 5e-4
    flow = po.Flow(initialRho=1.0, nu=nu, cs0=0.1, g3=0.8, useLES=les)
    lat = po.CpuLattice("port", x, y, z, flow, streaming, 4)
    cu = tb.ComputeUnit(x=x, y=y, z=z, nu=nu, cs0=0.1, g3=0.8, useLES=int(les),
                        streaming=tb.STREAMING_SIMPLE if streaming == "Simple" else tb.STREAMING_ESOTWIST)
    n = max(8, x * z // 2)
    mk = random_markers(tb, rng, n, x, y, z, planes=[0, y // 2, y - 1])
    lat.initialise(1.0)
    cu.initialise(1.0)
    lat.forcing(mk, ALPHA, BETA)
    cu.forcing(mk, ALPHA, BETA)
    compare(cu, lat, 0, "after initial forcing")
    for s in range(1, 9):
        mk = random_markers(tb, rng, n, x, y, z, planes=[0, y // 2, y - 1])
        lat.step(mk, ALPHA, BETA)
        cu.collision()
        cu.bounceBackBoundary()
        cu.streamingPush()
        cu.moments()
        cu.forcing(mk, ALPHA, BETA)
        assert cu.evenStep == lat.even_step
        compare(cu, lat, s, f"step {s}")
    cu.close()


def test_heavily_overlapping_markers_follow_list_order(gpu, port_oracle):
    """Dozens of markers on the same few cells: the level walk must apply
    them in list order exactly as the sequential reference does."""
    tb, po = gpu, port_oracle
    x, y, z = 8, 3, 8
    rng = np.random.default_rng(99)
    m = random_markers(tb, rng, 300, 3, 1, 3)
    m["i"] += 2
    m["k"] += 2
    m["j"] = 1
    lev, mx = tb.schedule_levels(m, x, y, z)
    assert mx > 50
    flow = po.Flow(nu=1e-3, useLES=True)
    lat = po.CpuLattice("port", x, y, z, flow, "Simple", 4)
    cu = tb.ComputeUnit(x=x, y=y, z=z, nu=1e-3, useLES=1, cs0=0.1)
    lat.initialise(1.0)
    cu.initialise(1.0)
    lat.forcing(m, ALPHA, BETA)
    cu.forcing(m, ALPHA, BETA)
    compare(cu, lat, 0, "overlap")
    for s in range(1, 4):
        lat.step(m, ALPHA, BETA)
        cu.collision()
        cu.forcing(m, ALPHA, BETA)
        compare(cu, lat, s, f"overlap step {s}")
    cu.close()


def _rushton_run(tb, po, edge, streaming, steps, kind, precision=4, with_gpu=True):
    nu = tb.nu_from_reynolds(7300.0, 0.1, edge // 6)
    rt = tb.RushtonTurbine(edge, edge, edge, tip_speed=0.1, startup_steps=30)
    flow = po.Flow(initialRho=1.0, nu=nu, cs0=0.1, g3=0.8, useLES=True)
    lat = po.CpuLattice(kind, edge, edge, edge, flow, streaming, precision)

    class _NoGpu:
        def __getattr__(self, name):
            return lambda *a, **k: None

    cu = tb.ComputeUnit(x=edge, y=edge, z=edge, nu=nu, cs0=0.1, g3=0.8, useLES=1,
                        streaming=tb.STREAMING_SIMPLE if streaming == "Simple" else tb.STREAMING_ESOTWIST) \
        if with_gpu else _NoGpu()
    angle = 0.0
    d0 = rt.increment(1)
    fixed, nonupd = rt.fixed(), rt.rotating_nonupdating(d0)
    mk = np.concatenate([fixed, nonupd, rt.rotating(angle, d0)])
    lat.initialise(1.0)
    cu.initialise(1.0)
    lat.forcing(mk, ALPHA, BETA)
    cu.forcing(mk, ALPHA, BETA)
    for step in range(2, steps + 2):          # main.cpp:336-455 (step starts at 1, incremented first)
        d = rt.increment(step)
        angle += d
        mk = np.concatenate([fixed, nonupd, rt.rotating(angle, d)])
        lat.step(mk, ALPHA, BETA)
        cu.collision()
        cu.forcing(mk, ALPHA, BETA)
    return cu, lat, steps


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
def test_rushton_tank_60_cubed_20_steps_vs_reference(gpu, ref_oracle, port_oracle, streaming):
    """The small configuration: 60^3, LES Cs=0.1, tip speed 0.1, Re=7300,
    rotating impeller, 20 steps, against the reference compiled in place
    (FP32) and the FP64 restatement.

    Tolerance (relative L2 over all interior cells after 20 steps):
      * GPU vs reference FP32: <= 1e-4 for rho, u, F and Nu;
      * GPU vs FP64: at most 2x the reference FP32's own error vs FP64 (the
        reference's FP32 rounding floor is ~2e-5 in u here).
    """
    tb, po = gpu, ref_oracle
    cu, lat, n = _rushton_run(tb, po, 60, streaming, 20, "ref")
    _, lat64, _ = _rushton_run(tb, po, 60, streaming, 20, "port", precision=8, with_gpu=False)
    mg = cu.read_moments().astype(np.float64)
    fg = cu.read_force().astype(np.float64)
    mr, fr = lat.get_moments(), lat.interior(lat.get_f())
    m64, f64 = lat64.get_moments(), lat64.interior(lat64.get_f())
    ug, ur, u64 = velocity(mg, fg), velocity(mr, fr), velocity(m64, f64)
    assert rel_l2(mg[..., 0], mr[..., 0]) <= 1e-4
    assert rel_l2(ug, ur) <= 1e-4
    assert rel_l2(fg, fr) <= 1e-4
    assert rel_l2(cu.read_nu(), lat.interior(lat.get_nu())) <= 1e-4
    assert rel_l2(ug, u64) <= 2.0 * rel_l2(ur, u64) + 1e-7
    assert rel_l2(mg[..., 0], m64[..., 0]) <= 2.0 * rel_l2(mr[..., 0], m64[..., 0]) + 1e-7
    cu.close()


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
def test_rushton_16_cubed_vs_golden_fixture(gpu, port_oracle, streaming):
    """Against the committed fixture tests/golden/rushton16_6steps.npz (the
    reference's own FP32 fields of a 16^3 Rushton tank after 6 steps, made by
    tests/golden/make_golden.py): the same tolerance as the 60^3 test,
    relative L2 <= 1e-4 for rho, u, F and Nu."""
    import os
    tb, po = gpu, port_oracle
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "rushton16_6steps.npz"))
    edge, steps = int(g["edge"]), int(g["steps"])
    cu, _, _ = _rushton_run(tb, po, edge, streaming, steps, "port")
    mg = cu.read_moments().astype(np.float64)
    fg = cu.read_force().astype(np.float64)
    assert rel_l2(mg[..., 0], g[f"{streaming}_rho"]) <= 1e-4
    assert rel_l2(velocity(mg, fg), g[f"{streaming}_u"]) <= 1e-4
    assert rel_l2(fg, g[f"{streaming}_F"]) <= 1e-4
    assert rel_l2(cu.read_nu(), g[f"{streaming}_Nu"]) <= 1e-4
    cu.close()


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
def test_step_variants_bit_identical(gpu, streaming):
    """1, 2 and 4 cells per thread run the same per-cell arithmetic: the
    states after several full steps must be bit-identical."""
    tb = gpu
    x, y, z = 10, 9, 37
    rng = np.random.default_rng(5)
    mk = random_markers(tb, rng, 60, x, y, z)
    states = []
    for vec in (1, 2, 4):
        cu = tb.ComputeUnit(x=x, y=y, z=z, nu=5e-4, cs0=0.1, useLES=1,
                            streaming=tb.STREAMING_SIMPLE if streaming == "Simple" else tb.STREAMING_ESOTWIST)
        cu.set_cells_per_thread(vec)
        cu.initialise(1.0)
        cu.forcing(mk, ALPHA, BETA)
        for _ in range(5):
            cu.collision()
            cu.forcing(mk, ALPHA, BETA)
        states.append((cu.debug_get_state(), cu.read_nu(), cu.read_force()))
        cu.close()
    for other in states[1:]:
        for a, b in zip(states[0], other):
            np.testing.assert_array_equal(a, b)


def test_marker_positions_bit_exact_on_device(gpu):
    """The touched flags equal the union of the stencils of the host list."""
    tb = gpu
    e = 32
    rt = tb.RushtonTurbine(e, e, e, tip_speed=0.1)
    mk = rt.forcing_list(0.4, rt.increment(1))
    cu = tb.ComputeUnit(x=e, y=e, z=e, nu=1e-3)
    cu.initialise(1.0)
    cu.forcing(mk, ALPHA, BETA)
    want = np.zeros((e, e, e), np.uint8)
    for k1 in (-1, 0, 1):
        for i1 in (-1, 0, 1):
            want[(mk["i"] + i1) % e, mk["j"], (mk["k"] + k1) % e] = 1
    np.testing.assert_array_equal(cu.read_touched(), want)
    cu.close()


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
def test_impeller_load_matches_oracle(gpu, port_oracle, streaming):
    """FP64 force and torque on the attached impeller (rotating-non-updating +
    rotating markers) against the oracle's per-marker spread sums."""
    tb, po = gpu, port_oracle
    e = 40
    rt = tb.RushtonTurbine(e, e, e, tip_speed=0.1)
    d = rt.increment(1)
    nu = tb.nu_from_reynolds(7300.0, 0.1, rt.blade_outer_radius())
    cu = tb.ComputeUnit(x=e, y=e, z=e, nu=nu, cs0=0.1, useLES=1,
                        streaming=tb.STREAMING_SIMPLE if streaming == "Simple" else tb.STREAMING_ESOTWIST)
    lat = po.CpuLattice("port", e, e, e, po.Flow(nu=nu, useLES=True), streaming, 4)
    cu.attach_rushton(rt, d, 0.0, d)
    mk = cu.read_markers()
    n_fixed = len(rt.fixed())
    cu.initialise(1.0)
    lat.initialise(1.0)
    angle = 0.0
    cu.forcing_resident(ALPHA, BETA)
    lat.forcing(mk, ALPHA, BETA)
    for _ in range(3):
        angle += d
        cu.rotate_impeller(angle, d)
        mk = cu.read_markers()
        cu.collision()
        cu.forcing_resident(ALPHA, BETA)
        lat.step(mk, ALPHA, BETA)
    load = cu.impeller_load()
    sums = lat.get_forcing_sums(len(mk))[n_fixed:]
    imp = mk[n_fixed:]
    ci = ck = (e - 1) / 2.0
    di = imp["i"] + imp["iCartFraction"].astype(np.float64) - ci
    dk = imp["k"] + imp["kCartFraction"].astype(np.float64) - ck
    f = -BETA * sums
    want = np.array([f[:, 0].sum(), f[:, 1].sum(), f[:, 2].sum(), (dk * f[:, 0] - di * f[:, 2]).sum(), len(imp)])
    assert load[4] == len(imp)
    scale = np.abs(f).sum()
    np.testing.assert_allclose(load[:3], want[:3], rtol=0, atol=2e-5 * scale)
    torque_scale = (np.abs(dk * f[:, 0]) + np.abs(di * f[:, 2])).sum()
    assert abs(load[3] - want[3]) <= 2e-5 * torque_scale
    cu.close()


def test_device_rotation_matches_host_generator(gpu):
    """Blade markers moved on the device are bit-identical to the host
    generator's markers at the same angle."""
    tb = gpu
    e = 48
    rt = tb.RushtonTurbine(e, e, e, tip_speed=0.1)
    d = rt.increment(1)
    cu = tb.ComputeUnit(x=e, y=e, z=e, nu=1e-3)
    cu.attach_rushton(rt, d, 0.0, d)
    n_rot = len(rt.rotating(0.0, d))
    for angle in (0.0, 0.1234, 1.0, 2.5, 6.1):
        cu.rotate_impeller(angle, d)
        dev = cu.read_markers()[-n_rot:]
        host = rt.rotating(angle, d)
        np.testing.assert_array_equal(dev.view(np.uint8), host.view(np.uint8))
    cu.close()


def test_shipped_debug_input_vs_reference(gpu, ref_oracle):
    """A unit made by tdlb_create from the reference's debug input
    (input_debug_gridx60_numSteps20.json: 60^3, initialRho 8, nu 0 as main.cpp's
    unit keeps it, cs0 0.12, LES off, Esotwist; its values are pinned against
    the shipped file by tests/test_input_file.py) against the reference's CPU
    unit built from the same values, with the file's impeller (uav 0.1,
    30 start-up steps): forcing, then 20 steps of main.cpp's sequence.
    Tolerance as the 60^3 test: relative L2 <= 1e-4 for rho, u and F."""
    import json
    from test_input_file import SHIPPED_DEBUG_INPUT as S
    tb, po = gpu, ref_oracle
    text = json.dumps({
        "GridParams": {"x": S["x"], "y": S["y"], "z": S["z"], "multiStep": S["multiStep"]},
        "FlowParams": {"initialRho": S["initialRho"], "reMNonDimensional": 7300.0, "uav": 0.1, "cs0": S["cs0"],
                       "g3": S["g3"], "nu": S["nu"], "alpha": S["alpha"], "beta": S["beta"], "useLES": S["useLES"],
                       "streaming": S["streaming"]},
    })
    cu = tb.ComputeUnit(params=text)
    flow = po.Flow(initialRho=S["initialRho"], nu=S["nu"], cs0=S["cs0"], g3=S["g3"], alpha=S["alpha"],
                   beta=S["beta"], useLES=S["useLES"])
    lat = po.CpuLattice("ref", S["x"], S["y"], S["z"], flow, S["streaming"], 4)
    rt = tb.RushtonTurbine(S["x"], S["y"], S["z"], tip_speed=0.1, startup_steps=30)
    d1 = rt.increment(1)
    fixed, nonupd = rt.fixed(), rt.rotating_nonupdating(d1)
    angle = 0.0
    mk = np.concatenate([fixed, nonupd, rt.rotating(angle, d1)])
    cu.initialise(S["initialRho"])
    lat.initialise(S["initialRho"])
    cu.forcing(mk, S["alpha"], S["beta"])
    lat.forcing(mk, S["alpha"], S["beta"])
    for step in range(2, 22):
        d = rt.increment(step)
        angle += d
        mk = np.concatenate([fixed, nonupd, rt.rotating(angle, d)])
        cu.collision()
        cu.bounceBackBoundary()
        cu.streamingPush()
        cu.moments()
        cu.forcing(mk, S["alpha"], S["beta"])
        lat.step(mk, S["alpha"], S["beta"])
    mg = cu.read_moments().astype(np.float64)
    fg = cu.read_force().astype(np.float64)
    mr, fr = lat.get_moments(), lat.interior(lat.get_f())
    assert np.isfinite(mr).all()
    assert rel_l2(mg[..., 0], mr[..., 0]) <= 1e-4
    assert rel_l2(velocity(mg, fg), velocity(mr, fr)) <= 1e-4
    assert rel_l2(fg, fr) <= 1e-4
    cu.close()
    lat.close()
