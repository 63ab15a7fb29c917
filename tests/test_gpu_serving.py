"""Serving form: requests admitted by free HBM (and a budget), resident
lattices, continuous batching into the persistent launch.

Stated tolerance: every request's final density and velocity fields in a
mix of overlapping requests equal those of the same request served alone
within 1e-6 relative L2 (the tanks share launches but no arithmetic, so in
practice they are bit-identical).
"""
import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# (id, edge, tip, Re, steps, storage, streaming)
MIX = [
    (1, 24, 0.10, 7300.0, 40, "fp32", "Simple"),
    (2, 32, 0.08, 2000.0, 25, "fp16", "Simple"),
    (3, 20, 0.12, 15000.0, 60, "fp32", "Simple"),
    (4, 28, 0.06, 1200.0, 33, "fp16", "Simple"),
    (5, 36, 0.09, 5000.0, 17, "fp32", "Simple"),
    (6, 24, 0.11, 9000.0, 44, "fp32", "Esotwist"),
]


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300)


def submit(server, req, fields=True):
    rid, edge, tip, re, steps, storage, streaming = req
    server.submit(rid, edge, tip, re, steps, storage=storage, streaming=streaming, fields=fields)


def collect(server, n, timeout=120.0):
    server.wait_idle(timeout)
    res = server.poll(1024)
    assert len(res) == n
    return {r["id"]: r for r in res}


def test_results_same_alone_and_in_mix(gpu):
    tb = gpu
    alone = {}
    with tb.Server(chunk_steps=8) as s:
        for req in MIX:
            submit(s, req)
            alone.update(collect(s, 1))
    with tb.Server(chunk_steps=8) as s:
        for req in MIX[:3]:
            submit(s, req)
        time.sleep(0.05)              # the rest arrive while the first ones run
        for req in MIX[3:]:
            submit(s, req)
        mix = collect(s, len(MIX))
        st = s.stats()
    for rid, r in mix.items():
        a = alone[rid]
        assert r["status"] == 0 and a["status"] == 0
        assert r["t_submit"] <= r["t_admit"] <= r["t_done"]
        for k in ("rho", "ux", "uy", "uz"):
            assert rel_l2(r["fields"][k], a["fields"][k]) <= 1e-6, (rid, k)
        assert abs(r["mass"] - a["mass"]) <= 1e-9 * abs(a["mass"])
        assert np.allclose(r["force"], a["force"], rtol=1e-6, atol=1e-12)
        edge = next(m[1] for m in MIX if m[0] == rid)
        assert abs(r["mass"] - edge ** 3) <= 1e-3 * edge ** 3
        assert r["power_number"] > 0
    # work overlapped: some requests were resident at the same time
    spans = sorted((r["t_admit"], r["t_done"]) for r in mix.values())
    assert any(spans[q + 1][0] < spans[q][1] for q in range(len(spans) - 1))
    assert st["completed"] == len(MIX) and st["lattice_updates"] == sum(m[1] ** 3 * m[4] for m in MIX)


def test_admission_waits_for_memory(gpu):
    tb = gpu
    need = tb.lattice_bytes(40, 40, 40)
    with tb.Server(hbm_budget=int(need * 1.5), chunk_steps=5) as s:
        s.submit(1, 40, 0.1, 3000.0, 30)
        s.submit(2, 40, 0.1, 3000.0, 30)
        res = collect(s, 2)
    a, b = res[1], res[2]
    assert a["status"] == 0 and b["status"] == 0
    assert b["t_admit"] >= a["t_done"]       # the second fitted only after the first left


def test_request_larger_than_budget_fails(gpu):
    tb = gpu
    with tb.Server(hbm_budget=tb.lattice_bytes(16, 16, 16)) as s:
        s.submit(9, 64, 0.1, 3000.0, 10)
        res = collect(s, 1)
    assert res[9]["status"] == -3            # TDLB_ENOMEM


def test_bad_request_rejected(gpu):
    tb = gpu
    with tb.Server() as s:
        with pytest.raises(tb.TdlbError):
            s.submit(1, 32, 0.1, 3000.0, 0)
        with pytest.raises(tb.TdlbError):
            s.submit(2, 4, 0.1, 3000.0, 10)


def test_submit_from_threads_and_close_with_work_pending(gpu):
    tb = gpu
    s = tb.Server(chunk_steps=4)
    threads = [threading.Thread(target=s.submit, args=(q, 24, 0.1, 3000.0, 400)) for q in range(8)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    time.sleep(0.02)
    s.close()                                # unfinished requests end, the worker stops


@pytest.mark.parametrize("streaming", ["Simple", "Esotwist"])
def test_served_request_vs_restatement(gpu, port_oracle, streaming):
    """One FP32 request (24^3, tip 0.1, Re 7300, 30 steps) served, against the
    CPU restatement of the same tank with the server's set-up (nu from
    calcNuAndRe_m of the blade radius, cs0 0.1, LES, impeller attached at
    increment(1) and advanced by increment(s) per step): density and velocity
    within 1e-4 relative L2, the single-tank parity tolerance."""
    tb, po = gpu, port_oracle
    edge, tip, re, steps = 24, 0.1, 7300.0, 30
    with tb.Server(chunk_steps=8) as s:
        s.submit(7, edge, tip, re, steps, storage="fp32", streaming=streaming, fields=True)
        r = collect(s, 1)[7]
    assert r["status"] == 0
    rt = tb.RushtonTurbine(edge, edge, edge, tip_speed=tip, startup_steps=0)
    nu = tb.nu_from_reynolds(re, tip, rt.blade_outer_radius())
    lat = po.CpuLattice("port", edge, edge, edge, po.Flow(initialRho=1.0, nu=nu, cs0=0.1, g3=0.8, useLES=True),
                        streaming, 4)
    d1 = rt.increment(1)
    lat.initialise(1.0)
    lat.forcing(rt.forcing_list(d1, d1, nonupdating_delta=d1), 0.97, 1.9)
    angle = d1
    for st in range(2, steps + 2):
        d = rt.increment(st)
        angle += d
        lat.step(rt.forcing_list(angle, d, nonupdating_delta=d1), 0.97, 1.9)
    m, f = lat.get_moments(), lat.interior(lat.get_f())
    lat.close()
    rho0 = m[..., 0]
    u0 = (m[..., 1:4] + 0.5 * f) / rho0[..., None]
    u = np.stack([r["fields"]["ux"], r["fields"]["uy"], r["fields"]["uz"]], axis=-1)
    assert rel_l2(r["fields"]["rho"], rho0) <= 1e-4
    assert rel_l2(u, u0) <= 1e-4
