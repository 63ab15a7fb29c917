"""Batched form: several tanks of uneven sizes advanced by one persistent
fused launch per step, per-tank immersed-boundary passes, device impeller
rotation from a per-step table, pairs of steps replayed from a CUDA graph.

Every tank of a batch must follow the same trajectory as the same tank run
alone through the single-lattice entry points with the reference's main-loop
sequence (main.cpp:409-454: rotate impeller, collision, forcing). Both run
the same device step bodies, so the stated tolerance is 1e-6 relative L2 on
velocity and density; graph replay against eager launches, and the
batched-launch shapes against each other, must agree bit for bit.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ALPHA, BETA = 0.97, 1.9

# (edge x, y, z, tip speed, Re, useLES, startup steps)
TANKS = [
    (24, 24, 24, 0.10, 7300.0, 1, 0),
    (36, 30, 36, 0.07, 2000.0, 0, 4),
    (20, 20, 20, 0.12, 15000.0, 1, 0),
    (33, 40, 33, 0.05, 1000.0, 1, 3),
]


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300)


def tank_config(tb, spec, streaming, storage):
    x, y, z, tip, re, les, startup = spec
    rt = tb.RushtonTurbine(x, y, z, tip_speed=tip, startup_steps=startup)
    nu = tb.nu_from_reynolds(re, tip, rt.blade_outer_radius())
    cfg = dict(x=x, y=y, z=z, nu=nu, cs0=0.1, useLES=les, initialRho=1.0, streaming=streaming, storage=storage)
    return rt, cfg


def prepare(cu, rt):
    d1 = rt.increment(1)
    cu.attach_rushton(rt, d1, d1, d1)
    cu.initialise(1.0)
    cu.forcing_resident(ALPHA, BETA)


def run_alone(tb, spec, streaming, storage, steps):
    rt, cfg = tank_config(tb, spec, streaming, storage)
    cu = tb.ComputeUnit(**cfg)
    prepare(cu, rt)
    if storage != "fp32":
        # a tank of a batch keeps no 16-bit residual box and steps one cell
        # per thread: compare like with like
        cu.set_residual_box(0, 0, 0, 0, 0, 0)
        cu.set_cells_per_thread(1)
        prepare(cu, rt)
    angle = rt.increment(1)
    for s in range(2, steps + 2):
        d = rt.increment(s)
        angle += d
        cu.rotate_impeller(angle, d)
        cu.collision()
        cu.forcing_resident(ALPHA, BETA)
    out = cu.read_velocity_density(), cu.read_force(), cu.read_touched()
    cu.close()
    return out


def make_batch(tb, streaming, storage, specs=TANKS):
    rts, cfgs = zip(*(tank_config(tb, s, streaming, storage) for s in specs))
    b = tb.Batch(list(cfgs))
    for cu, rt in zip(b.tanks, rts):
        prepare(cu, rt)
    return b


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
@pytest.mark.parametrize("storage", ["fp32", "fp16"])
@pytest.mark.parametrize("steps", [1, 6, 7])
def test_batch_matches_tanks_alone(gpu, streaming, storage, steps):
    tb = gpu
    with make_batch(tb, streaming, storage) as b:
        b.run(steps, ALPHA, BETA)
        got = [((cu.read_velocity_density()), cu.read_force(), cu.read_touched()) for cu in b.tanks]
    for spec, ((rho, u), F, touched) in zip(TANKS, got):
        (rho0, u0), F0, t0 = run_alone(tb, spec, streaming, storage, steps)
        assert rel_l2(u, u0) <= 1e-6, spec
        assert rel_l2(rho, rho0) <= 1e-6, spec
        assert rel_l2(F, F0) <= 1e-5, spec
        assert np.array_equal(touched, t0), spec


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
def test_graph_replay_equals_eager(gpu, streaming):
    tb = gpu
    res = []
    for graph in (True, False):
        with make_batch(tb, streaming, "fp32") as b:
            b.run(3, ALPHA, BETA, graph=graph)   # one eager step, one pair, ...
            b.run(4, ALPHA, BETA, graph=graph)   # ... then a run of two pairs
            res.append([cu.read_moments() for cu in b.tanks])
    for a, c in zip(*res):
        assert np.array_equal(a, c)


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
def test_chunked_runs_equal_one_run(gpu, streaming):
    """Runs of 10, 10, 3 and 10 steps (graphs captured by the first run and
    replayed by the later ones, one-pair graphs and an odd last step) leave
    every tank where one run of 33 steps does, bit for bit."""
    tb = gpu
    res = []
    for chunks in ([10, 10, 3, 10], [33]):
        with make_batch(tb, streaming, "fp32") as b:
            for c in chunks:
                b.run(c, ALPHA, BETA)
            res.append([(cu.read_moments(), cu.read_force()) for cu in b.tanks])
    for (m0, f0), (m1, f1) in zip(*res):
        assert np.array_equal(m0, m1)
        assert np.array_equal(f0, f1)


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
def test_batch_shapes_agree(gpu, streaming):
    tb = gpu
    res = []
    for shape in [(1, 128, 4), (2, 256, 2), (4, 128, 8), (4, 256, 1), (1, 128, 0)]:
        with make_batch(tb, streaming, "fp32") as b:
            b.set_shape(*shape)
            assert b.shape() == shape
            b.run(5, ALPHA, BETA)
            res.append([cu.read_moments() for cu in b.tanks])
    for other in res[1:]:
        for a, c in zip(res[0], other):
            assert np.array_equal(a, c)


def test_autotune_then_run(gpu):
    tb = gpu
    with make_batch(tb, "Esotwist", "fp32") as b:
        ms = b.autotune(trials=2)
        assert ms > 0
        v, t, bps = b.shape()
        assert v in (1, 2, 4) and t in (128, 256) and 0 <= bps <= 16
        for cu in b.tanks:   # the timed launches changed the fields
            cu.initialise(1.0)
            cu.forcing_resident(ALPHA, BETA)
        b.run(4, ALPHA, BETA)
        rho, u = b.tanks[0].read_velocity_density()
        assert np.isfinite(u).all() and np.isfinite(rho).all()


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
def test_adopted_tank_matches_tank_alone(gpu, streaming):
    """A tank set up on its own stream while a batch is running (the serving
    form's admission) joins the batch and then follows the trajectory it
    follows alone; the tanks already there carry on."""
    tb = gpu
    with make_batch(tb, streaming, "fp32", TANKS[:2]) as b:
        b.run(3, ALPHA, BETA)
        rt, cfg = tank_config(tb, TANKS[2], streaming, "fp32")
        cu = tb.ComputeUnit(**cfg)
        prepare(cu, rt)
        assert b.adopt(cu) is cu and len(b) == 3
        b.run(5, ALPHA, BETA)
        (rho, u), F = cu.read_velocity_density(), cu.read_force()
        with pytest.raises(tb.TdlbError):
            b.adopt(cu)               # already the batch's
        cu.close()                    # a view now: the batch still owns the tank
        assert len(b) == 3
        b.run(1, ALPHA, BETA)
    (rho0, u0), F0, _ = run_alone(tb, TANKS[2], streaming, "fp32", 5)
    assert rel_l2(u, u0) <= 1e-6
    assert rel_l2(rho, rho0) <= 1e-6
    assert rel_l2(F, F0) <= 1e-5


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
def test_detached_tank_continues_alone(gpu, streaming):
    """A tank detached from a batch after 5 steps (the serving form's
    retirement) keeps its state, continues through the single-lattice entry
    points for 2 more steps and ends where 7 steps alone end; the batch
    carries on with the other tanks."""
    tb = gpu
    spec = TANKS[1]
    with make_batch(tb, streaming, "fp32", TANKS[:3]) as b:
        b.run(5, ALPHA, BETA)
        cu = b.detach(1)
        assert len(b) == 2
        b.run(3, ALPHA, BETA)
        rt, _ = tank_config(tb, spec, streaming, "fp32")
        angle = rt.increment(1)
        for s in range(2, 7):
            angle += rt.increment(s)
        for s in range(7, 9):
            d = rt.increment(s)
            angle += d
            cu.rotate_impeller(angle, d)
            cu.collision()
            cu.forcing_resident(ALPHA, BETA)
        (rho, u), F = cu.read_velocity_density(), cu.read_force()
        cu.close()                    # owned again: destroys the tank
    (rho0, u0), F0, _ = run_alone(tb, spec, streaming, "fp32", 7)
    assert rel_l2(u, u0) <= 1e-6
    assert rel_l2(rho, rho0) <= 1e-6
    assert rel_l2(F, F0) <= 1e-5


def test_batch_rejects_mixed_schemes(gpu):
    tb = gpu
    cfgs = [dict(x=8, y=8, z=8, nu=1e-3), dict(x=8, y=8, z=8, nu=1e-3, streaming="Esotwist")]
    with pytest.raises(tb.TdlbError, match="streaming"):
        tb.Batch(cfgs)
    with pytest.raises(tb.TdlbError, match="initialised"):
        with tb.Batch([dict(x=8, y=8, z=8, nu=1e-3)]) as b:
            b.run(1, ALPHA, BETA)


def oracle_tank(po, tb, spec, streaming, steps):
    """The same tank on the restatement (bit-identical to the reference's CPU
    unit), with the batch's impeller schedule: markers attached at angle
    d1 = increment(1), then per step s the angle advanced by increment(s)."""
    x, y, z, tip, re, les, startup = spec
    rt = tb.RushtonTurbine(x, y, z, tip_speed=tip, startup_steps=startup)
    nu = tb.nu_from_reynolds(re, tip, rt.blade_outer_radius())
    lat = po.CpuLattice("port", x, y, z, po.Flow(initialRho=1.0, nu=nu, cs0=0.1, g3=0.8, useLES=bool(les)),
                        streaming, 4)
    d1 = rt.increment(1)
    lat.initialise(1.0)
    lat.forcing(rt.forcing_list(d1, d1, nonupdating_delta=d1), ALPHA, BETA)
    angle = d1
    for s in range(2, steps + 2):
        d = rt.increment(s)
        angle += d
        lat.step(rt.forcing_list(angle, d, nonupdating_delta=d1), ALPHA, BETA)
    m, f = lat.get_moments(), lat.interior(lat.get_f())
    rho = m[..., 0]
    u = (m[..., 1:4] + 0.5 * f) / rho[..., None]
    o = lat.interior(lat.get_o())
    lat.close()
    return rho, u, f, o


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
def test_batched_tanks_vs_restatement(gpu, port_oracle, streaming):
    """Tanks of a batch (16^3, 24^3 and 32^3, LES, 10 steps) against the CPU
    restatement directly, not only against the same tanks run alone: rho,
    u and F within 1e-4 relative L2 (the tolerance of the single-tank parity
    tests), touched flags bit-exact."""
    tb, po = gpu, port_oracle
    specs = [(16, 16, 16, 0.10, 7300.0, 1, 0), (24, 24, 24, 0.08, 3000.0, 1, 0), (32, 32, 32, 0.12, 15000.0, 1, 0)]
    steps = 10
    with make_batch(tb, streaming, "fp32", specs) as b:
        b.run(steps, ALPHA, BETA)
        got = [(cu.read_velocity_density(), cu.read_force(), cu.read_touched()) for cu in b.tanks]
    for spec, ((rho, u), F, touched) in zip(specs, got):
        rho0, u0, F0, t0 = oracle_tank(po, tb, spec, streaming, steps)
        assert rel_l2(rho, rho0) <= 1e-4, spec
        assert rel_l2(u, u0) <= 1e-4, spec
        assert rel_l2(F, F0) <= 1e-4, spec
        assert np.array_equal(touched.astype(bool), t0.astype(bool)), spec
