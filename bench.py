#!/usr/bin/env python3
"""Throughput benchmark of the B200 lattice Boltzmann time step.

Workload (default): the stirred tank at scale -- a 400^3 FP32 lattice,
Rushton turbine (T = 400, D = T/3, 6 blades, 4 baffles), Eggels-Somers
collision with Smagorinsky LES (Cs = 0.1), tip speed 0.1, Re = 20000,
Simple (A/B) streaming, rotating impeller. `--workload esotwist` runs the
same tank with single-buffer esoteric-twist streaming.

One "step" = the reference's main-loop step (main.cpp:409-454): impeller
update, collision + streaming + moments (one fused kernel), immersed-boundary
forcing. Metric: MLUPS = interior cells x steps / s.

  value   device-resident steps (markers rotated on the device), CUDA events
          on the library's stream, barrier + synchronize on both sides, max
          over ranks; the 9.6 GB lattice is far larger than L2, so no flush.
  e2e     the public C-ABI driven the way main.cpp drives the reference: per
          step the host generates the blade markers at the new angle, copies
          them from pinned memory (H2D), runs collision + forcing, and reads
          back the FP64 impeller load (D2H), reading step s's load after
          queueing step s+1; wall-clock, synchronized at both ends.
  roofline  the fused step kernel: 152 algorithmic bytes per cell (18
          populations read + written, Nu read + written) / its average
          CUDA-event duration, against the measured copy bandwidth.
  cpu_baseline  the reference's own CPU ComputeUnit (compiled in place into
          oracle/_ref) on a bounded sample of the same workload.

`--impl reference` times the reference's CPU implementation instead: every
host thread advances its own reference ComputeUnit on a 400 x h x 400 slab
through the impeller plane of the same tank (h = 16 planes, 8 when K + W
exceeds 100, so that the run ends within a few minutes), one reference step
per "step", K timed steps after W warm-up steps. That process loads only the
reference harness (oracle/_ref), which also carries the project's marker
generator.

Multi-GPU: `torchrun --nproc-per-node N bench.py --gpus N` runs one replica
per GPU (independent tanks, no collective: weak scaling).
"""
from __future__ import annotations

import argparse
import csv
import io
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

EDGE = 400
RE = 20000.0
TIP = 0.1
ALPHA, BETA = 0.97, 1.9
PROFILE_TRAFFIC = os.path.join(ROOT, "profiles", "traffic_per_cell.txt")


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(workload: str):
    """DRAM bytes per cell of the fused kernel from the committed ncu summary."""
    if not os.path.exists(PROFILE_TRAFFIC):
        return None
    with open(PROFILE_TRAFFIC) as f:
        for line in f:
            if line.startswith(workload + ":"):
                return float(line.split(":", 1)[1].split()[0])
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        rows = []
        for r in csv.reader(io.StringIO(self.out or "")):
            if len(r) < 9:
                continue
            try:
                rows.append([x.strip() for x in r])
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[c - 5] for r in rows for c in range(5, 9) if r[c].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------- our arm

def make_unit(tb, workload: str, edge: int, device: int, storage: str = "fp32"):
    rt = tb.RushtonTurbine(edge, edge, edge, tip_speed=TIP, startup_steps=0)
    nu = tb.nu_from_reynolds(RE, TIP, rt.blade_outer_radius())
    streaming = tb.STREAMING_ESOTWIST if workload == "esotwist" else tb.STREAMING_SIMPLE
    cu = tb.ComputeUnit(x=edge, y=edge, z=edge, nu=nu, cs0=0.1, g3=0.8, useLES=1, initialRho=1.0,
                        streaming=streaming, device=device, storage=storage)
    return cu, rt, nu


def run_ours(args, rank, world, device):
    import torch
    import tdlbcpp_b200 as tb

    torch.cuda.set_device(device)
    edge = args.edge
    cu, rt, nu = make_unit(tb, args.workload, edge, device, args.storage)
    stream = torch.cuda.ExternalStream(cu.stream, device=device)
    dth = rt.increment(1)
    cu.attach_rushton(rt, dth, 0.0, dth)
    cu.initialise(1.0)
    cu.forcing_resident(ALPHA, BETA)          # main.cpp:305
    n_markers = len(cu.read_markers())
    n_rot = len(rt.rotating(0.0, dth))
    cells = edge ** 3
    angle = 0.0

    def device_step():
        nonlocal angle
        angle += dth
        cu.rotate_impeller(angle, dth)
        cu.collision()
        cu.forcing_resident(ALPHA, BETA)

    cu.set_overlap(args.overlap)
    for _ in range(args.warmup):
        device_step()
    cu.synchronize()
    try:
        zone = cu.read_zone() if args.overlap else None
    except tb.TdlbError:
        zone = None   # the zone covers most of this lattice: steps are not split

    # ---- value: device-resident steps. The library brackets every step-kernel
    # launch with CUDA events on the stream it runs on (a split step is two
    # launches on two streams); t1 follows a join of both streams.
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier(world)
    cu.synchronize()
    torch.cuda.synchronize()
    cu.kernel_time()
    cu.set_kernel_timing(True)
    launches0 = cu.kernel_launches()
    with ClockSampler(device) as clk:
        t0.record(stream)
        for s in range(args.steps):
            device_step()
        cu.join()
        t1.record(stream)
        cu.synchronize()
        torch.cuda.synchronize()
    barrier(world)
    launches = cu.kernel_launches() - launches0
    kernel_total_ms, kernel_n = cu.kernel_time()
    cu.set_kernel_timing(False)
    ms = t0.elapsed_time(t1)
    kernel_ms = kernel_total_ms / args.steps
    ms = max_over_ranks(ms, world)
    kernel_ms_max = max_over_ranks(kernel_ms, world)

    # ---- e2e: host-driven steps through the C ABI. Per step the host
    # generates the blades at the step's angle into pinned memory and uploads
    # them (tdlb_set_rotating_markers), the step runs, and its FP64 impeller
    # load comes back to pinned host memory. The host prepares step s+1's
    # blades while the device runs step s (their upload is queued after the
    # load of step s, which still needs step s's blades) and reads step s's
    # load after queueing step s+1, so the device never waits for the host.
    pinned = torch.empty(n_rot * tb.MARKER_DTYPE.itemsize, dtype=torch.uint8, pin_memory=True)
    host_rot = np.frombuffer(pinned.numpy(), dtype=tb.MARKER_DTYPE)
    load = torch.empty((2, 5), dtype=torch.float64, pin_memory=True)   # steps alternate between the rows
    load_np = load.numpy()
    got = [torch.cuda.Event(), torch.cuda.Event()]
    spec = rt.spec
    # at least 50 steps and 0.6 s of wall clock, so that one host hiccup
    # cannot move the figure by much
    k_e2e = max(50, args.steps, int(math.ceil(600.0 / max(ms / args.steps, 1e-3))))
    loads = []

    def upload_next():
        nonlocal angle
        angle += dth
        n = tb.ctypes.c_size_t()
        rc = cu.lib.tdlb_rushton_rotating(tb.ctypes.byref(spec), angle, dth, tb._p(host_rot), n_rot, tb.ctypes.byref(n))
        assert rc == 0 and n.value == n_rot
        cu.set_rotating_markers(host_rot)

    def e2e_steps(k):
        # the device always has the next step queued: step s is queued, the
        # host prepares step s+1's blades, and only then waits for the load
        # of step s-1 (two pinned rows, so no step's copy overwrites a load
        # the host has not read)
        upload_next()
        for s in range(k):
            cu.collision()
            cu.forcing_resident(ALPHA, BETA)
            cu.impeller_load_async(load[s % 2].data_ptr())
            got[s % 2].record(stream)
            if s + 1 < k:
                upload_next()
            if s >= 1:
                got[(s - 1) % 2].synchronize()
                loads.append(load_np[(s - 1) % 2].copy())
        got[(k - 1) % 2].synchronize()
        loads.append(load_np[(k - 1) % 2].copy())

    # the fields after the timed steps; then the e2e run starts again from
    # rest (initialise + forcing, main.cpp:261-305), so that it stays within
    # the step count the Simple wall rule keeps finite
    red_timed = cu.reduce_fp64()
    cu.initialise(1.0)
    cu.forcing_resident(ALPHA, BETA)
    e2e_steps(2)
    barrier(world)
    cu.synchronize()
    loads.clear()
    w0 = time.perf_counter()
    e2e_steps(k_e2e)
    cu.synchronize()
    w1 = time.perf_counter()
    barrier(world)
    load_np = loads[-1]
    e2e_s = max_over_ranks(w1 - w0, world)
    red = cu.reduce_fp64()
    cu.close()

    result = {
        "value_mlups": world * cells * args.steps / (ms / 1e3) / 1e6,
        "ms_per_step": ms / args.steps,
        "kernel_ms": kernel_ms_max,
        "e2e_mlups": world * cells * k_e2e / e2e_s / 1e6,
        "e2e_steps": k_e2e,
        "h2d": n_rot * tb.MARKER_DTYPE.itemsize,
        "d2h": 5 * 8,
        "clocks": clk.summary(),
        "n_markers": n_markers,
        "n_rot": n_rot,
        "nu": nu,
        "load": load_np.tolist(),
        "fields_finite_end": bool(np.isfinite(red).all() and np.isfinite(load_np).all()),
        "fields_finite_after_timed": bool(np.isfinite(red_timed).all()),
        "steps_before_timed_check": args.warmup + args.steps,
        "e2e_steps_from_rest": k_e2e + 2,
        "mass_drift_timed": float(red_timed[0] / cells - 1.0),
        "mass_drift_end": float(red[0] / cells - 1.0),
        "launches": launches,
        "step_launches": kernel_n,
        "inner_fraction": None if zone is None else float(zone.mean()),
    }
    return result


# ---------------------------------------------------------------- batched form

BATCH_EDGES = (32, 48, 64, 96, 128)
BATCH_SEED = 20261203
BATCH_TANKS = 64


def draw_batched_tanks(n=BATCH_TANKS, seed=BATCH_SEED):
    """Tank list of the batched workload: per tank, in this order, the edge
    uniform over BATCH_EDGES, tip speed U[0.05, 0.12], Re log-uniform on
    [1e3, 2e4], all from numpy's default_rng(seed)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        edge = int(rng.choice(BATCH_EDGES))
        tip = float(rng.uniform(0.05, 0.12))
        re = float(np.exp(rng.uniform(np.log(1e3), np.log(2e4))))
        out.append((edge, tip, re))
    return out


def batched_configs(tb, tanks, storage="fp32", streaming="Esotwist"):
    rts, cfgs = [], []
    for edge, tip, re in tanks:
        rt = tb.RushtonTurbine(edge, edge, edge, tip_speed=tip, startup_steps=0)
        nu = tb.nu_from_reynolds(re, tip, rt.blade_outer_radius())
        rts.append(rt)
        cfgs.append(dict(x=edge, y=edge, z=edge, nu=nu, cs0=0.1, g3=0.8, useLES=1, initialRho=1.0,
                         streaming=streaming, storage=storage))
    return rts, cfgs


def prepare_tank(cu, rt):
    d = rt.increment(1)
    cu.attach_rushton(rt, d, d, d)
    cu.initialise(1.0)
    cu.forcing_resident(ALPHA, BETA)          # main.cpp:305


def run_batched(args, rank, world, device):
    """The batched form: 64 tanks in one batch, timed over K batched steps;
    beside it the same tanks stepped one after another in the plain form."""
    import torch
    import tdlbcpp_b200 as tb

    torch.cuda.set_device(device)
    tanks = draw_batched_tanks()
    rts, cfgs = batched_configs(tb, tanks, storage=args.storage)
    cells = sum(e ** 3 for e, _, _ in tanks)
    b = tb.Batch(cfgs, device=device)
    stream = torch.cuda.ExternalStream(b.stream(), device=device)
    for cu, rt in zip(b.tanks, rts):
        prepare_tank(cu, rt)
    b.run(4, ALPHA, BETA)
    fused_ms = b.autotune(trials=5)
    shape = b.shape()
    for cu, rt in zip(b.tanks, rts):              # autotuning changed the fields
        prepare_tank(cu, rt)
    # warm-up: W steps, then one untimed run of the timed run's length, so
    # that the CUDA graphs that length replays (four step pairs per graph,
    # one-pair graphs for the rest) are captured before the clock starts
    b.run(args.warmup, ALPHA, BETA)
    b.run(args.steps, ALPHA, BETA)
    b.synchronize()

    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = b.kernel_launches()
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(device) as clk:
        t0.record(stream)
        b.run(args.steps, ALPHA, BETA)
        t1.record(stream)
        b.synchronize()
        torch.cuda.synchronize()
    barrier(world)
    ms = max_over_ranks(t0.elapsed_time(t1), world)
    launches = b.kernel_launches() - l0

    # fused batched launch alone, timed on the batch stream after the run
    fused = []
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.run(1, ALPHA, BETA)
        e1.record(stream)
        b.synchronize()
        fused.append(e0.elapsed_time(e1))

    # e2e: public API with host buffers -- chunks of 10 steps, then every
    # tank's FP64 impeller load read back to pinned host memory (queued on
    # the batch's stream, one wait per chunk)
    chunk = 10
    n_chunks = max(5, args.steps // chunk, int(math.ceil(600.0 / max(chunk * ms / args.steps, 1e-3))))
    load_t = torch.empty((len(tanks), 5), dtype=torch.float64, pin_memory=True)
    load = load_t.numpy()
    b.synchronize()
    w0 = time.perf_counter()
    for _ in range(n_chunks):
        b.run(chunk, ALPHA, BETA)
        for t, cu in enumerate(b.tanks):
            cu.impeller_load_async(load_t.data_ptr() + t * 5 * 8)
        b.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - w0, world)
    finite = bool(np.isfinite(load).all())
    b.close()

    # the same tanks in the plain form, one after another
    seq_ms = 0.0
    k_seq = max(5, min(20, args.steps // 10))
    for (edge, tip, re), rt, cfg in zip(tanks, rts, cfgs):
        cu = tb.ComputeUnit(device=device, **cfg)
        prepare_tank(cu, rt)
        st = torch.cuda.ExternalStream(cu.stream, device=device)
        angle, s = rt.increment(1), 1

        def plain_step():
            nonlocal angle, s
            s += 1
            d = rt.increment(s)
            angle += d
            cu.rotate_impeller(angle, d)
            cu.collision()
            cu.forcing_resident(ALPHA, BETA)

        for _ in range(3):
            plain_step()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        cu.synchronize()
        e0.record(st)
        for _ in range(k_seq):
            plain_step()
        e1.record(st)
        cu.synchronize()
        seq_ms += e0.elapsed_time(e1) / k_seq
        cu.close()

    return {
        "value_mlups": world * cells * args.steps / (ms / 1e3) / 1e6,
        "ms_per_step": ms / args.steps,
        "kernel_ms": fused_ms,
        "step_ms_single": statistics.median(fused),
        "e2e_mlups": world * cells * chunk * n_chunks / e2e_s / 1e6,
        "e2e_steps": chunk * n_chunks,
        "d2h": len(tanks) * 5 * 8 / chunk,
        "seq_mlups": world * cells / (seq_ms / 1e3) / 1e6,
        "seq_steps": k_seq,
        "cells": cells,
        "shape": shape,
        "launches": launches,
        "clocks": clk.summary(),
        "tanks": len(tanks),
        "fields_finite": finite,
    }


# ---------------------------------------------------------------- precision form

PREC_STEPS = 2000
PREC_ORACLE_EDGE = 120
PREC_STREAMING = "Esotwist"   # the Simple wall rule diverges within these step counts


def power_number(torque, omega, D):
    """|torque * omega| / (N^3 D^5), N = omega / 2 pi, rho = 1 (lattice units)."""
    n = omega / (2.0 * math.pi)
    return abs(torque * omega) / (n ** 3 * D ** 5)


def gpu_precision_run(tb, edge, storage, steps, device, timed=False):
    import torch
    rt = tb.RushtonTurbine(edge, edge, edge, tip_speed=TIP, startup_steps=0)
    nu = tb.nu_from_reynolds(RE, TIP, rt.blade_outer_radius())
    cu = tb.ComputeUnit(x=edge, y=edge, z=edge, nu=nu, cs0=0.1, g3=0.8, useLES=1, initialRho=1.0, storage=storage,
                        streaming=PREC_STREAMING, device=device)
    d1 = rt.increment(1)
    cu.attach_rushton(rt, d1, d1, d1)
    cu.initialise(1.0)
    cu.forcing_resident(ALPHA, BETA)
    mass0 = cu.reduce_fp64()[0]
    st = torch.cuda.ExternalStream(cu.stream, device=device)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    angle = d1
    cu.synchronize()
    t0.record(st)
    for s in range(2, steps + 2):
        d = rt.increment(s)
        angle += d
        cu.rotate_impeller(angle, d)
        cu.collision()
        cu.forcing_resident(ALPHA, BETA)
    cu.join()
    t1.record(st)
    cu.synchronize()
    ms = t0.elapsed_time(t1)
    rho, u = cu.read_velocity_density()
    red = cu.reduce_fp64()
    load = cu.impeller_load()
    cu.close()
    return {"u": u, "rho": rho, "mass0": mass0, "mass": red[0], "torque": load[3], "ms": ms,
            "omega": d1, "D": rt.spec.impeller_diameter or edge / 3.0}


def oracle_precision_run(tb, po, edge, steps, threads):
    rt = tb.RushtonTurbine(edge, edge, edge, tip_speed=TIP, startup_steps=0)
    nu = tb.nu_from_reynolds(RE, TIP, rt.blade_outer_radius())
    flow = po.Flow(initialRho=1.0, nu=nu, cs0=0.1, g3=0.8, alpha=ALPHA, beta=BETA, useLES=True)
    po.load("port").tdlbo_set_threads(threads)
    lat = po.CpuLattice("port", edge, edge, edge, flow, PREC_STREAMING, 8)
    d1 = rt.increment(1)
    n_fixed = len(rt.fixed())
    lat.initialise(1.0)
    lat.forcing(rt.forcing_list(d1, d1, nonupdating_delta=d1), ALPHA, BETA)
    angle = d1
    t = time.perf_counter()
    mk = None
    for s in range(2, steps + 2):
        d = rt.increment(s)
        angle += d
        mk = rt.forcing_list(angle, d, nonupdating_delta=d1)
        lat.step(mk, ALPHA, BETA)
    secs = time.perf_counter() - t
    m = lat.get_moments()
    f = lat.interior(lat.get_f())
    rho = m[..., 0]
    u = (m[..., 1:4] + 0.5 * f) / rho[..., None]
    sums = lat.get_forcing_sums(len(mk))[n_fixed:]
    imp = mk[n_fixed:]
    ci = ck = (edge - 1) / 2.0
    di = imp["i"] + imp["iCartFraction"].astype(np.float64) - ci
    dk = imp["k"] + imp["kCartFraction"].astype(np.float64) - ck
    fx, fz = -BETA * sums[:, 0], -BETA * sums[:, 2]
    torque = float(np.sum(dk * fx - di * fz))
    lat.close()
    return {"u": u, "rho": rho, "mass0": float(edge ** 3), "mass": float(rho.sum()), "torque": torque,
            "seconds": secs, "omega": d1, "D": edge / 3.0}


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def run_precision(args, rank, world, device):
    """FP16 / BF16 deviation storage against the FP64 oracle (120^3) and
    against the plain FP32 GPU form (400^3), both after PREC_STEPS steps."""
    import torch
    import tdlbcpp_b200 as tb
    from oracle import pyoracle as po

    torch.cuda.set_device(device)
    steps = args.steps if args.steps != 500 else PREC_STEPS
    out = {"steps": steps, "oracle_edge": PREC_ORACLE_EDGE}
    # FP64 oracle at 120^3 (host threads), then the GPU forms at 120^3
    threads = max(1, min(64, os.cpu_count() or 1))
    ref = oracle_precision_run(tb, po, PREC_ORACLE_EDGE, steps, threads)
    np_ref = power_number(ref["torque"], ref["omega"], ref["D"])
    out["oracle"] = {"threads": threads, "seconds": ref["seconds"], "mass_drift": ref["mass"] / ref["mass0"] - 1.0,
                     "power_number": np_ref, "finite": bool(np.isfinite(ref["u"]).all())}
    small = {}
    for storage in ("fp32", "fp16", "bf16"):
        g = gpu_precision_run(tb, PREC_ORACLE_EDGE, storage, steps, device)
        small[storage] = g
        npn = power_number(g["torque"], g["omega"], g["D"])
        out[f"{storage}_vs_fp64_120"] = {
            "u_rel_l2": rel(g["u"], ref["u"]), "rho_rel_l2": rel(g["rho"], ref["rho"]),
            "mass_drift": g["mass"] / g["mass0"] - 1.0, "power_number": npn,
            "power_number_rel_err": abs(npn - np_ref) / abs(np_ref) if np_ref else None}
    # the 400^3 forms: throughput, and the 16-bit forms against FP32
    big = {}
    for storage in ("fp32", "fp16", "bf16"):
        g = gpu_precision_run(tb, args.edge, storage, steps, device, timed=True)
        big[storage] = {"mlups": args.edge ** 3 * steps / (g["ms"] / 1e3) / 1e6, "ms_per_step": g["ms"] / steps,
                        "mass_drift": g["mass"] / g["mass0"] - 1.0,
                        "power_number": power_number(g["torque"], g["omega"], g["D"]), "u": g["u"]}
    for storage in ("fp16", "bf16"):
        big[storage]["u_rel_l2_vs_fp32"] = rel(big[storage]["u"], big["fp32"]["u"])
    for storage in big:
        big[storage].pop("u")
    out["gpu_400"] = big
    return out


def report_precision(args, rank, world, local, config):
    res = run_precision(args, rank, world, local)
    if rank != 0:
        return 0
    peak, peak_kind = measured_peak()
    fp16 = res["gpu_400"]["fp16"]
    achieved = 80 * args.edge ** 3 / (fp16["ms_per_step"] / 1e3) / 1e9
    config = dict(config, results=res)
    line = {
        "metric": "MLUPS", "value": fp16["mlups"], "unit": "MLUPS", "n_gpus": world, "steps": res["steps"],
        "warmup": 0, "ms_per_step": fp16["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp16 storage, fp32 arithmetic", "data": "synthetic", "config": config,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "kernel": "whole step (rotate + fused step + IBM), 80 B/cell",
                     "bytes_per_cell": 80, "traffic": None},
        "fp32_mlups": res["gpu_400"]["fp32"]["mlups"], "bf16_mlups": res["gpu_400"]["bf16"]["mlups"],
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- serving form

SERVE_EDGES = (48, 64, 96, 128, 192, 256)
SERVE_SEED = 20261204
SERVE_RATE = 20.0          # requests per second
SERVE_TOTAL = 2000
SERVE_TIP = 0.1
# Esotwist (periodic in the reference): the reference's Simple wall rule lets
# small tanks diverge after a few hundred steps, Esotwist tanks stay finite
SERVE_STREAMING = "Esotwist"


def draw_serving_requests(n=SERVE_TOTAL, seed=SERVE_SEED):
    """The request stream of the serving workload: Poisson arrivals at
    SERVE_RATE per second; per request, in this order, the exponential gap to
    its arrival, the edge uniform over SERVE_EDGES, the step count uniform on
    [500, 5000], Re log-uniform on [1e3, 2e4] and the storage, FP32 or FP16
    with probability 1/2 each, all from numpy's default_rng(seed)."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    for q in range(n):
        t += float(rng.exponential(1.0 / SERVE_RATE))
        edge = int(rng.choice(SERVE_EDGES))
        steps = int(rng.integers(500, 5001))
        re = float(np.exp(rng.uniform(np.log(1e3), np.log(2e4))))
        storage = "fp16" if rng.uniform() < 0.5 else "fp32"
        out.append({"id": q, "arrival": t, "edge": edge, "steps": steps, "re": re, "storage": storage})
    return out


def plain_fields(tb, edge, re, steps, device):
    """One request solved alone in the plain FP32 form (the per-request
    error reference): host-driven rotate / collision / forcing steps."""
    rt = tb.RushtonTurbine(edge, edge, edge, tip_speed=SERVE_TIP, startup_steps=0)
    nu = tb.nu_from_reynolds(re, SERVE_TIP, rt.blade_outer_radius())
    cu = tb.ComputeUnit(x=edge, y=edge, z=edge, nu=nu, cs0=0.1, g3=0.8, useLES=1, initialRho=1.0, device=device,
                        streaming=SERVE_STREAMING)
    d1 = rt.increment(1)
    cu.attach_rushton(rt, d1, d1, d1)
    cu.initialise(1.0)
    cu.forcing_resident(ALPHA, BETA)
    angle = d1
    for s in range(2, steps + 2):
        d = rt.increment(s)
        angle += d
        cu.rotate_impeller(angle, d)
        cu.collision()
        cu.forcing_resident(ALPHA, BETA)
    rho, u = cu.read_velocity_density()
    cu.close()
    return rho, u


def run_serving(args, rank, world, device):
    """The serving form on a prefix of the seeded request stream: requests
    are submitted at their arrival times from a host thread; the native
    server admits, batches and retires them."""
    import torch
    import tdlbcpp_b200 as tb

    torch.cuda.set_device(device)
    reqs = draw_serving_requests()[:args.requests]
    # per-request error: the two smallest FP16 requests and the smallest FP32 one
    fp16 = sorted((r for r in reqs if r["storage"] == "fp16"), key=lambda r: r["edge"] ** 3 * r["steps"])[:2]
    fp32 = sorted((r for r in reqs if r["storage"] == "fp32"), key=lambda r: r["edge"] ** 3 * r["steps"])[:1]
    checked = {r["id"] for r in fp16 + fp32}
    server = tb.Server(device=device, max_active=64, chunk_steps=args.chunk)
    t_start = time.perf_counter()

    def feeder():
        for r in reqs:
            delay = r["arrival"] - (time.perf_counter() - t_start)
            if delay > 0:
                time.sleep(delay)
            server.submit(r["id"], r["edge"], SERVE_TIP, r["re"], r["steps"], storage=r["storage"],
                          streaming=SERVE_STREAMING, fields=r["id"] in checked)

    barrier(world)
    with ClockSampler(device) as clk:
        th = threading.Thread(target=feeder)
        th.start()
        th.join()
        server.wait_idle(3600.0)
    results = server.poll(len(reqs) + 8)
    st = server.stats()
    why = server.lib.tdlb_server_last_error(server.h).decode()
    server.close()
    bad = [r for r in results if r["status"] != 0]
    if bad:
        raise RuntimeError(f"{len(bad)} serving requests failed, first status {bad[0]['status']}: {why}")
    lat = np.array([r["t_done"] - r["t_submit"] for r in results])
    t0 = min(r["t_submit"] for r in results)
    t1 = max(r["t_done"] for r in results)
    lu = float(sum(r["cells"] * r["steps"] for r in results))
    errors = []
    for r in results:
        if r["id"] not in checked:
            continue
        q = next(x for x in reqs if x["id"] == r["id"])
        rho0, u0 = plain_fields(tb, q["edge"], q["re"], q["steps"], device)
        f = r["fields"]
        u = np.stack([f["ux"], f["uy"], f["uz"]], axis=-1)
        eu = float(np.linalg.norm((u - u0).ravel()) / max(np.linalg.norm(u0.ravel()), 1e-300))
        er = float(np.linalg.norm((f["rho"] - rho0).ravel()) / np.linalg.norm(rho0.ravel()))
        errors.append({"id": q["id"], "edge": q["edge"], "steps": q["steps"], "storage": q["storage"],
                       "u_rel_l2_vs_plain_fp32": eu, "rho_rel_l2_vs_plain_fp32": er})
    bytes_done = sum(r["cells"] * r["steps"] * (152 if next(x for x in reqs if x["id"] == r["id"])["storage"] == "fp32"
                                                 else 80) for r in results)
    return {
        "value_mlups": world * lu / (t1 - t0) / 1e6,
        "busy_mlups": st["lattice_updates"] / st["busy_s"] / 1e6 if st["busy_s"] > 0 else None,
        "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
        "mean_s": float(lat.mean()), "span_s": t1 - t0, "lattice_updates": lu,
        "achieved_gbs": bytes_done / st["busy_s"] / 1e9 if st["busy_s"] > 0 else None,
        "chunks": st["chunks"], "requests": len(results), "errors": errors, "clocks": clk.summary(),
        "ms_per_step": None,
    }


def report_serving(args, rank, world, local, config):
    res = run_serving(args, rank, world, local)
    if rank != 0:
        return 0
    peak, peak_kind = measured_peak()
    config = dict(config, p50_latency_s=res["p50_s"], p99_latency_s=res["p99_s"], mean_latency_s=res["mean_s"],
                  span_s=res["span_s"], device_busy_mlups=res["busy_mlups"], chunks=res["chunks"],
                  per_request_error=res["errors"])
    line = {
        "metric": "MLUPS", "value": res["value_mlups"], "unit": "MLUPS", "n_gpus": world,
        "steps": int(res["lattice_updates"]), "warmup": 0, "ms_per_step": None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "fp32/fp16", "data": "synthetic", "config": config,
        "roofline": {"bound": "hbm", "achieved": res["achieved_gbs"], "peak": peak, "unit": "GB/s",
                     "frac": None if res["achieved_gbs"] is None else res["achieved_gbs"] / peak,
                     "peak_kind": peak_kind, "kernel": "whole serving step (stepping wall time)",
                     "bytes_per_cell": "152 (fp32) / 80 (fp16)", "traffic": None},
        "e2e": {"value": res["value_mlups"], "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                "note": "submit to result through the public server API, wall clock"},
        "latency_p50_s": res["p50_s"], "latency_p99_s": res["p99_s"],
        "clocks": res["clocks"],
    }
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------- reference arm

def slab_markers(rt, j0, height, angle, dth):
    m = rt.forcing_list(angle, dth, nonupdating_delta=dth)
    m = m[(m["j"] >= j0) & (m["j"] < j0 + height)].copy()
    m["j"] -= j0
    return m


def reference_height(steps, warmup):
    """Slab height of the reference sample: 16 planes, 8 for long runs, so
    that --steps K --warmup W ends within a few minutes on the host cores."""
    return 16 if steps + warmup <= 100 else 8


def reference_sample(steps, warmup, threads, edge=EDGE, height=16):
    """Every thread advances its own reference ComputeUnit (FP32, Simple,
    LES) on an edge x height x edge slab through the impeller plane.

    Only the reference harness (oracle/_ref/libtdlb_ref.so) is loaded: the
    marker lists come from the project's generator compiled into that
    harness and nu from the reference's own calcNuAndRe_m, so this process
    never maps the B200 library."""
    from oracle import pyoracle as po

    rt = po.RefRushton(edge, edge, edge, tip_speed=TIP, startup_steps=0)
    nu = po.ref_nu(RE, TIP, rt.blade_outer_radius())
    dth = rt.increment(1)
    j0 = int(round(edge / 3.0)) - height // 2
    flow = po.Flow(initialRho=1.0, nu=nu, cs0=0.1, g3=0.8, alpha=ALPHA, beta=BETA, useLES=True)
    lats = [po.CpuLattice("ref", edge, height, edge, flow, "Simple", 4, tmpdir="/tmp") for _ in range(threads)]
    mk = slab_markers(rt, j0, height, 0.0, dth)
    for L in lats:
        L.initialise(1.0)
        L.forcing(mk, ALPHA, BETA)
    angle = 0.0
    times = []
    for s in range(warmup + steps):
        angle += dth
        mk = slab_markers(rt, j0, height, angle, dth)
        ths = [threading.Thread(target=L.step, args=(mk, ALPHA, BETA)) for L in lats]
        t = time.perf_counter()
        for th in ths:
            th.start()
        for th in ths:
            th.join()
        if s >= warmup:
            times.append(time.perf_counter() - t)
    for L in lats:
        L.close()
    cells = threads * edge * height * edge
    total = sum(times)
    return {"value": cells * len(times) / total / 1e6, "cores": threads, "seconds": total,
            "sample": f"{threads} x reference ComputeUnit<float,...,Simple,CPU> on a {edge}x{height}x{edge} slab "
                      f"through the impeller plane, {len(times)} timed step(s) each after {warmup} warm-up step(s)"}


def host_threads(edge=EDGE, height=16):
    """Threads for the reference sample: every host core, bounded by the RAM
    one reference slab takes (~100 B per cell with ghosts) and capped at 64."""
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    try:
        avail = os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")
        per = (edge + 2) * (height + 2) * (edge + 2) * 110
        n = min(n, max(1, int(avail * 0.5 // per)))
    except (ValueError, OSError):
        pass
    return max(1, min(n, 64))


# ---------------------------------------------------------------- plumbing

_PG = None


_DEVICE = "cuda"


def init_dist(args, backend=None):
    """One process per GPU (RANK / LOCAL_RANK / WORLD_SIZE from torchrun):
    NCCL on GPUs; gloo where no GPU is visible (the CPU tests of the
    multi-rank helpers)."""
    global _PG, _DEVICE
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        _DEVICE = "cuda" if backend == "nccl" else "cpu"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        _PG = dist
    return rank, world, local


def barrier(world):
    if world > 1 and _PG is not None:
        _PG.barrier()


def max_over_ranks(x, world):
    """The slowest rank's time: every multi-GPU number is timed on each
    device and reduced with MAX."""
    if world > 1 and _PG is not None:
        import torch
        t = torch.tensor([float(x)], device=_DEVICE)
        _PG.all_reduce(t, op=_PG.ReduceOp.MAX)
        return float(t.item())
    return float(x)


BATCH_ERROR_STEPS = 1000


def batched_error(tb, tanks, storage, device, count=2, steps=BATCH_ERROR_STEPS):
    """Velocity error of the `count` smallest tanks of the batched workload
    after `steps` batched steps (the workload's step count), against the FP64
    CPU restatement of each tank (host threads) with the batch's impeller
    schedule: relative L2 per tank."""
    from oracle import pyoracle as po
    picked = sorted(range(len(tanks)), key=lambda t: tanks[t][0])[:count]
    sub = [tanks[t] for t in picked]
    rts, cfgs = batched_configs(tb, sub, storage=storage)
    with tb.Batch(cfgs, device=device) as b:
        for cu, rt in zip(b.tanks, rts):
            prepare_tank(cu, rt)
        b.run(steps, ALPHA, BETA)
        got = [cu.read_velocity_density()[1].astype(np.float64) for cu in b.tanks]
    po.load("port").tdlbo_set_threads(max(1, min(64, os.cpu_count() or 1)))
    out = []
    for (edge, tip, re), rt, cfg, u in zip(sub, rts, cfgs, got):
        lat = po.CpuLattice("port", edge, edge, edge, po.Flow(initialRho=1.0, nu=cfg["nu"], cs0=0.1, g3=0.8,
                                                              alpha=ALPHA, beta=BETA, useLES=True), "Esotwist", 8)
        d1 = rt.increment(1)
        lat.initialise(1.0)
        lat.forcing(rt.forcing_list(d1, d1, nonupdating_delta=d1), ALPHA, BETA)
        angle = d1
        for s in range(2, steps + 2):
            d = rt.increment(s)
            angle += d
            lat.step(rt.forcing_list(angle, d, nonupdating_delta=d1), ALPHA, BETA)
        m, f = lat.get_moments(), lat.interior(lat.get_f())
        lat.close()
        uref = (m[..., 1:4] + 0.5 * f) / m[..., 0:1]
        out.append({"edge": edge, "tip": tip, "re": re, "steps": steps, "u_rel_l2_vs_fp64": rel(u, uref)})
    return out


def report_batched(args, rank, world, local, config):
    res = run_batched(args, rank, world, local)
    if rank != 0:
        return 0
    peak, peak_kind = measured_peak()
    bpc = 152 if args.storage == "fp32" else 80
    achieved = bpc * res["cells"] / (res["kernel_ms"] / 1e3) / 1e9
    v, nt, bps = res["shape"]
    if args.storage != "fp32" and not args.no_cpu_baseline:
        import tdlbcpp_b200 as tb
        config = dict(config, error_vs_fp64=batched_error(tb, draw_batched_tanks(), args.storage, local))
    config = dict(config, shape={"cells_per_thread": v, "threads": nt, "blocks_per_sm": bps},
                  sequential_plain_mlups=res["seq_mlups"], sequential_steps_per_tank=res["seq_steps"],
                  single_step_ms=res["step_ms_single"])
    line = {
        "metric": "MLUPS", "value": res["value_mlups"], "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup + args.steps, "ms_per_step": res["ms_per_step"], "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32" if args.storage == "fp32" else f"fp32 arithmetic, {args.storage} storage",
        "data": "synthetic", "config": config,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "kernel": "k_batch_step", "bytes_per_cell": bpc,
                     "kernel_ms": res["kernel_ms"], "traffic": None},
        "e2e": {"value": res["e2e_mlups"], "unit": "MLUPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": res["d2h"], "steps": res["e2e_steps"]},
        "gpu_launches": res["launches"],
        "clocks": res["clocks"],
        "fields_finite": res["fields_finite"],
    }
    if world == 1 and not args.no_cpu_baseline:
        r = reference_sample(3, 1, host_threads())
        line["cpu_baseline"] = {"value": r["value"], "unit": "MLUPS", "cores": r["cores"], "kind": "reference",
                                "sample": r["sample"] + " (per-cell rate of the same step)"}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["simple", "esotwist", "batched", "serving", "precision"], default="simple")
    ap.add_argument("--requests", type=int, default=64, help="serving: prefix of the request stream to serve")
    ap.add_argument("--chunk", type=int, default=100, help="serving: steps per batched chunk")
    ap.add_argument("--edge", type=int, default=EDGE)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--overlap", action="store_true",
                    help="simple/esotwist: split steps (outer cells overlap the previous forcing pass)")
    ap.add_argument("--storage", choices=["fp32", "fp16", "bf16"], default="fp32",
                    help="simple/esotwist: population storage (16-bit forms store deviations from the rest weights)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3   # timing rule: at least 3 warm-up steps
    if args.workload == "precision":
        workload = f"precision-{args.edge}^3-esotwist-fp16-bf16-les"
        config = {"workload": workload, "grid": [args.edge] * 3, "oracle_grid": [PREC_ORACLE_EDGE] * 3,
                  "streaming": PREC_STREAMING, "storage": "fp16/bf16 deviations f_i - w_i*rho0, fp32 arithmetic",
                  "fp64": "mass/momentum sums, impeller torque, power number", "re": RE, "tip_speed": TIP,
                  "collision": "EgglesSomers+LES(cs0=0.1)", "ibm": "Rushton turbine, rotating"}
    elif args.workload == "serving":
        workload = f"serving-{args.requests}-of-{SERVE_TOTAL}-requests"
        config = {"workload": workload, "requests": args.requests, "stream_total": SERVE_TOTAL, "seed": SERVE_SEED,
                  "rate_per_s": SERVE_RATE, "edges": list(SERVE_EDGES), "steps": [500, 5000], "re": [1e3, 2e4],
                  "storage": "fp32/fp16 50/50", "tip_speed": SERVE_TIP, "chunk_steps": args.chunk,
                  "streaming": SERVE_STREAMING,
                  "sample": f"the first {args.requests} requests of the seeded {SERVE_TOTAL}-request stream",
                  "l2": "lattices > L2 (no flush needed)"}
    elif args.workload == "batched":
        tanks = draw_batched_tanks()
        workload = f"batched-{len(tanks)}-tanks-esotwist-{args.storage}-les"
        config = {"workload": workload, "tanks": len(tanks), "edges": [t[0] for t in tanks],
                  "cells": sum(t[0] ** 3 for t in tanks), "seed": BATCH_SEED,
                  "draw": "edge U{32,48,64,96,128}, tip U[0.05,0.12], Re log-U[1e3,2e4] per tank, in that order",
                  "streaming": "Esotwist", "collision": "EgglesSomers+LES(cs0=0.1)", "ibm": "Rushton turbine, rotating",
                  "l2": "lattices > L2 every step (no flush needed)"}
    else:
        workload = f"rushton-{args.edge}^3-{args.workload}-{args.storage}-les"
        config = {"workload": workload, "grid": [args.edge] * 3, "streaming": args.workload.capitalize(),
                  "collision": "EgglesSomers+LES(cs0=0.1)", "re": RE, "tip_speed": TIP,
                  "ibm": "Rushton turbine, rotating", "l2": "lattice > L2 every step (no flush needed)"}

    rank, world, local = init_dist(args)

    if args.impl == "reference":
        if rank != 0:
            return 0
        nthr = host_threads()
        steps, warm = args.steps, args.warmup
        h = reference_height(steps, warm)
        r = reference_sample(steps, warm, nthr, height=h)
        line = {"metric": "MLUPS", "value": r["value"], "unit": "MLUPS", "n_gpus": args.gpus, "steps": steps,
                "warmup": warm, "ms_per_step": r["seconds"] / steps * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "fp32", "data": "synthetic", "config": config,
                "impl": "reference",
                "cpu_baseline": {"value": r["value"], "unit": "MLUPS", "cores": r["cores"], "kind": "reference",
                                 "sample": r["sample"]},
                "e2e": {"value": r["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return 0

    if args.workload == "batched":
        return report_batched(args, rank, world, local, config)
    if args.workload == "serving":
        return report_serving(args, rank, world, local, config)
    if args.workload == "precision":
        return report_precision(args, rank, world, local, config)

    res = run_ours(args, rank, world, local)
    if rank != 0:
        return 0
    peak, peak_kind = measured_peak()
    cells = args.edge ** 3
    bpc = 152 if args.storage == "fp32" else 80
    achieved = bpc * cells / (res["kernel_ms"] / 1e3) / 1e9
    traffic_pc = profile_traffic(workload)
    line = {
        "metric": "MLUPS", "value": res["value_mlups"], "unit": "MLUPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": res["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32" if args.storage == "fp32" else f"fp32 arithmetic, {args.storage} storage",
        "data": "synthetic", "config": config,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "kernel": "k_step_simple" if args.workload == "simple" else "k_step_esotwist",
                     "bytes_per_cell": bpc, "kernel_ms": res["kernel_ms"],
                     "traffic": None if traffic_pc is None else traffic_pc * cells},
        "e2e": {"value": res["e2e_mlups"], "unit": "MLUPS", "h2d_bytes_per_step": res["h2d"],
                "d2h_bytes_per_step": res["d2h"], "steps": res["e2e_steps"],
                # the e2e leg restarts from rest and runs at least 0.6 s; the
                # Simple scheme's wall rule diverges after a few hundred steps
                # from rest, as the reference's does, so its fields may end
                # non-finite there
                "steps_from_rest": res["e2e_steps_from_rest"], "fields_finite_at_end": res["fields_finite_end"],
                "mass_drift_at_end": res["mass_drift_end"]},
        "gpu_launches": res["launches"],
        "clocks": res["clocks"],
        "markers": res["n_markers"],
        "split_step": {"on": res["inner_fraction"] is not None, "inner_cell_fraction": res["inner_fraction"],
                       "step_launches_per_step": res["step_launches"] / args.steps},
        # the fields and the FP64 mass after the warm-up and timed steps
        "fields_finite": res["fields_finite_after_timed"],
        "steps_from_rest_at_check": res["steps_before_timed_check"],
        "mass_drift": res["mass_drift_timed"],
    }
    if world == 1 and not args.no_cpu_baseline:
        r = reference_sample(3, 1, host_threads())
        line["cpu_baseline"] = {"value": r["value"], "unit": "MLUPS", "cores": r["cores"], "kind": "reference",
                                "sample": r["sample"]}
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
