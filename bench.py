#!/usr/bin/env python
"""Benchmark: plain forward TTI elastic RSG modelling on one B200 per rank.

Workload (the demo shape of the reference, seeded synthetic salt-like model):
nz=1126 nx=7872 dx=dz=10 m, ealThick=60 (E=65, padded grid 1256 x 8002 =
10,050,512 cells), free surface, one 12 Hz Ricker source at the surface centre,
7872 receivers at z=2, dt=0.8 ms. A "step" is one time step (velocity and
stress half-steps over the padded grid); the metric is Gcell-updates/s over
the padded grid (Nz * Nx per step), summed over ranks (one shot per GPU, weak
scaling, no collective on the data path).

Arms:
  default            the CUDA library through the C ABI (inputs resident in HBM
                     for `value`; host buffers and the whole public-API call
                     sequence for `e2e`)
  --impl reference   the reference's own OpenMP C build (oracle/_ref) on the
                     host cores, a bounded number of steps of the same workload
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "tti-fdmodeling_b200"))
import synthetic  # noqa: E402

MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM = 6650.0
# Compulsory bytes per cell-update with the reference storage layout (state
# read+written once, per-cell parameters read once).
ALG_BYTES_STEP = {"coordinate_rotation": 84, "tensor_rotation": 104, "bond_transformation": 76}
# Compulsory bytes per cell of each half-step kernel when the two half-steps
# run as separate kernels (each re-reads the state the other wrote).
ALG_BYTES_HALF = {
    "coordinate_rotation": {"velocity": 48, "stress": 64},   # v: 3 sig + 2 v + 5 par + 2 w; s: 2 v + 3 sig + 8 par + 3 w
    "tensor_rotation": {"velocity": 40, "stress": 88},       # s: 2 v + 3 tau + 7 par + 6 w
    "bond_transformation": {"velocity": 40, "stress": 68},   # s: 2 v + 3 sig + 9 par + 3 w
}

WORKLOAD = dict(nz=1126, nx=7872, dx=10.0, dz=10.0, dt=0.0008, fpeak=12.0, ealThick=60, freesurface=1, stype=1,
                seistype=3, mt=1, wsave=2, savew=0, snap_sample=1250, mode=1, scalar=1.0, energy=0)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def peaks():
    try:
        d = json.load(open(MEASURED_PEAKS))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- inputs
_MODEL = None


def model():
    global _MODEL
    if _MODEL is None:
        _MODEL = synthetic.salt_model(WORKLOAD["nz"], WORKLOAD["nx"], seed=1)
    return _MODEL


def geometry(rank: int):
    nx, nt = WORKLOAD["nx"], None
    sx = nx // 2 + 12 * rank  # one shot per rank, 120 m apart
    gx = np.arange(nx, dtype=np.int32)
    gz = np.full(nx, 2, np.int32)
    return sx, 2, gx, gz


# ---------------------------------------------------------------- our arm
def workload_config(variant: str, world: int) -> dict:
    """The `config` block of both arms (same keys, so the two lines compare)."""
    E = WORKLOAD["ealThick"] + 5
    Nz, Nx = WORKLOAD["nz"] + 2 * E, WORKLOAD["nx"] + 2 * E
    return {"workload": f"plain forward, {variant}, salt-like synthetic {WORKLOAD['nz']}x{WORKLOAD['nx']} "
                        f"(padded {Nz}x{Nx}), freesurface, 12 Hz Ricker at the surface centre, "
                        f"{WORKLOAD['nx']} receivers at z=2",
            "variant": variant, "nz": WORKLOAD["nz"], "nx": WORKLOAD["nx"], "Nz": Nz, "Nx": Nx, "cells": Nz * Nx,
            "dt": WORKLOAD["dt"], "parallelism": f"shots x{world}",
            "l2": "inputs larger than L2 (>= 16 arrays x 41 MB per step)"}


def traffic_per_launch(variant: str):
    """DRAM bytes per launch of the two half-step kernels from the committed ncu
    summary (scaled from a narrower capture, as the file says), or None."""
    tfile = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        d = json.load(open(tfile))
        return d.get(variant), d.get("_note", "")
    except Exception:
        return None, ""


def measure_plain(variant, K, W, nprof, rank, world, local_rank, clock_window_s=1.0):
    """Device-resident throughput of the plain path for one formulation: K timed
    steps (CUDA events on the library's stream, max over ranks), the per-phase
    split over `nprof` more steps, and the step-level roofline. The clock
    sampler runs over the timed region and then over `clock_window_s` seconds
    of the same steps (the timed region alone is too short for nvidia-smi)."""
    import ttifd

    m = model()
    pads = synthetic.padded(m, WORKLOAD["ealThick"])
    sx, sz, gx, gz = geometry(rank)
    extra = 4000
    cfg = dict(WORKLOAD, variant=variant, nt=W + K + nprof + extra)
    wav = synthetic.ricker(cfg["nt"], cfg["dt"], cfg["fpeak"])
    with ttifd.Modeling(device=local_rank, **cfg) as h:
        h.upload_model(*pads)
        h.set_source([sx], [sz], wav[None, :])
        for k in (0, 1, 2):
            h.set_receivers(k, gx, gz)
        cells = h.Nz * h.Nx
        h.reset()
        h.step(W)
        dist_barrier()
        l0 = h.kernel_launches
        with ClockSampler(local_rank) as clk:
            h.step(K)
            ms = h.elapsed_ms
            launches = h.kernel_launches - l0
            # the same steps again, untimed, so that the sampler sees the load
            t0, left = time.perf_counter(), extra
            while time.perf_counter() - t0 < clock_window_s and left > 0:
                n = min(left, 500)
                h.step(n)
                left -= n
        ms_max = dist_max(ms)
        pv, ps, po = h.profile_steps(nprof)
        Nz, Nx, E = h.Nz, h.Nx, h.E
    peak, src = peaks()
    step_ms = ms_max / K
    alg = ALG_BYTES_STEP[variant]
    achieved = alg * cells / (step_ms / 1e3) / 1e9
    interior = (Nx - 10) * (Nz - 5 - E)  # free surface: rows [E, Nz-5)
    traffic, tnote = traffic_per_launch(variant)
    kernels = {}
    for name, t in (("velocity", pv), ("stress", ps)):
        if t == 0.0:
            continue
        kms = t / nprof
        b = ALG_BYTES_HALF[variant][name] * interior
        k = {"kernel": f"k_{name}_tiled<{variant}>", "alg_bytes_per_cell": ALG_BYTES_HALF[variant][name],
             "cells_per_launch": interior, "launch_ms": kms, "achieved_GBps": b / (kms / 1e3) / 1e9,
             "frac": b / (kms / 1e3) / 1e9 / peak}
        if traffic and name in traffic:
            k["ncu_dram_bytes"] = traffic[name]
            k["ncu_frac"] = traffic[name] / (kms / 1e3) / 1e9 / peak
        kernels[name] = k
    step_traffic = sum(traffic[n] for n in ("velocity", "stress")) if traffic and ps > 0 else None
    roof = {"bound": "hbm", "kernel": "time step (velocity + stress half-steps + column pass)",
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_source": src,
            "alg_bytes_per_cell_update": alg, "cells_per_step": cells, "step_ms": step_ms,
            "traffic": step_traffic,
            "traffic_note": ("DRAM bytes per step (velocity + stress launches) from ncu, scaled by interior cells "
                             "from a narrower capture: " + tnote) if step_traffic else None,
            "kernels": kernels,
            "phase_ms_per_step": {"velocity": pv / nprof, "stress": ps / nprof, "other": po / nprof}}
    return {"value": cells * K * world / (ms_max / 1e3) / 1e9, "ms_per_step": step_ms, "cells": cells,
            "launches": launches, "roofline": roof, "clocks": clk.summary()}


SNAP_KINDS = {0: 0, 1: 2, 2: 1, 3: 3, 4: 2, 5: 2}  # wsave -> snapshot kinds per snapshot step


def measure_e2e(variant, K, rank, world, local_rank, reps=3):
    """The whole public-API sequence from host buffers: create, upload of the
    physical model (tti_upload_model_physical: the rims are filled on the
    device) + device precompute, geometry, K steps with snapshots delivered to the host,
    traces fetched, destroy (wall clock, max over ranks). The model, trace and
    snapshot buffers are page-locked host arrays (tti_host_alloc), allocated
    and filled once outside the timed region, as a service that models shot
    after shot keeps them; every copy between them and the device is inside
    it. One untimed pass, then `reps` timed passes; the median pass is
    reported (all walls listed)."""
    import ttifd

    m = model()
    phys = m.arrays()  # the physical model; tti_upload_model_physical fills the rims on the device
    pinned = [ttifd.host_empty(a.shape) for a in phys]
    for d, a in zip(pinned, phys):
        d[...] = a
    sx, sz, gx, gz = geometry(rank)
    cfg_e = dict(WORKLOAD, variant=variant, nt=K)
    wav_e = synthetic.ricker(K, cfg_e["dt"], cfg_e["fpeak"])
    nts = (K - 1) // cfg_e["mt"] + 1
    trace_out = [ttifd.host_empty((gx.size, nts)) for _ in range(3)]
    pad = 0 if WORKLOAD["savew"] == 0 else 2 * (WORKLOAD["ealThick"] + 5)  # savew = 0: the physical area
    nk = SNAP_KINDS[WORKLOAD["wsave"]]
    snap_buf = ttifd.host_empty(nk * (WORKLOAD["nz"] + pad) * (WORKLOAD["nx"] + pad)) if nk else None

    def one():
        dist_barrier()
        phases = {}
        snaps = []
        t0 = time.perf_counter()
        with ttifd.Modeling(device=local_rank, **cfg_e) as he:
            phases["create"] = time.perf_counter() - t0
            he.upload_model_physical(*pinned)
            phases["upload"] = time.perf_counter() - t0 - sum(phases.values())
            he.set_source([sx], [sz], wav_e[None, :])
            for k in (0, 1, 2):
                he.set_receivers(k, gx, gz)
            if snap_buf is not None:
                he.set_snapshot_buffer(snap_buf)
            phases["geometry"] = time.perf_counter() - t0 - sum(phases.values())
            # the snapshot reaches host memory; the callback sees it in place
            # (as a C caller's callback does) and takes its size
            he.run(lambda it, kind, a: snaps.append(a.nbytes), copy=False)
            phases["run"] = time.perf_counter() - t0 - sum(phases.values())
            trs = [he.fetch_traces(k, out=trace_out[k]) for k in (0, 1, 2)]
            phases["fetch"] = time.perf_counter() - t0 - sum(phases.values())
            cells = he.Nz * he.Nx
        t = dist_max(time.perf_counter() - t0)
        phases["destroy"] = t - sum(phases.values())
        d2h = sum(snaps) + sum(x.nbytes for x in trs)
        return t, phases, cells, d2h

    one()  # untimed: first use of the snapshot and transpose kernels in the process
    runs = sorted((one() for _ in range(reps)), key=lambda r: r[0])
    t_e2e, phases, cells, d2h = runs[len(runs) // 2]
    h2d = sum(a.nbytes for a in phys) + wav_e.nbytes + 3 * 2 * gx.nbytes
    return {"value": cells * K * world / t_e2e / 1e9, "unit": "Gcell/s", "h2d_bytes_per_step": h2d / K,
            "d2h_bytes_per_step": d2h / K, "wall_s": t_e2e, "walls_s": [r[0] for r in runs], "phases_s": phases,
            "host_buffers": "page-locked (tti_host_alloc), allocated once outside the timed region",
            "includes": "tti_create..tti_destroy: physical-model upload (rims padded on the device) + device "
                        "precompute, geometry, K steps, "
                        "snapshots to host, traces; median of %d passes after one untimed pass" % reps}


def run_ours(args, rank, world, local_rank):
    variant = args.variant
    K, W = args.steps, args.warmup
    p = measure_plain(variant, K, W, args.profile_steps, rank, world, local_rank)
    e2e = measure_e2e(variant, K, rank, world, local_rank)
    line = {"metric": "Gcell-updates/s", "value": p["value"], "unit": "Gcell/s", "n_gpus": world, "steps": K,
            "warmup": W, "ms_per_step": p["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": workload_config(variant, world),
            "roofline": p["roofline"], "e2e": e2e, "gpu_launches": p["launches"], "clocks": p["clocks"]}
    # the same rate over the physical grid (nz * nx, without the absorbing rims)
    phys = WORKLOAD["nz"] * WORKLOAD["nx"] / p["cells"]
    line["value_physical"] = p["value"] * phys
    if not args.no_variants:
        # the other two formulations on the same workload, so the line carries all three
        line["variants"] = {}
        for v in ALG_BYTES_STEP:
            if v == variant:
                continue
            q = measure_plain(v, K, W, args.profile_steps, rank, world, local_rank, clock_window_s=0.5)
            q["e2e"] = measure_e2e(v, K, rank, world, local_rank)
            q["config"] = workload_config(v, world)
            q["value_physical"] = q["value"] * phys
            line["variants"][v] = q
    return line


# ---------------------------------------------------------------- batched arm
BATCH_WORKLOAD = dict(nz=1126, nx=3000, x0=2436, dx=10.0, dz=10.0, dt=0.0008, fpeak=10.0, ealThick=50,
                      freesurface=1, stype=1, seistype=1, mt=1, wsave=0, savew=0, mode=1, scalar=1.0, energy=0)


def run_batched(args, local_rank):
    """Many shots of one model through tti_batch_* (one launch per half-step for
    all shots, the loop in CUDA-graph replays) against one shot of the same
    model through the plain path. Shots 120 m apart along the surface of the
    nx=3000 crop (columns 2436..5435) of the salt-like model, 3000 receivers
    per shot at z=2, 10 Hz, ealThick=50, free surface."""
    import ttifd

    variant, S, K, W = args.variant, args.batch_shots, args.batch_steps, args.warmup
    bw = dict(BATCH_WORKLOAD)
    x0 = bw.pop("x0")
    m = synthetic.crop(model(), x0, bw["nx"]) if WORKLOAD["nx"] >= x0 + bw["nx"] else \
        synthetic.salt_model(bw["nz"], bw["nx"], seed=1)
    pads = synthetic.padded(m, bw["ealThick"])
    cfg = dict(bw, variant=variant, nt=W + K)
    wav = synthetic.ricker(cfg["nt"], cfg["dt"], cfg["fpeak"])[None, :]
    gx = np.arange(bw["nx"], dtype=np.int32)
    gz = np.full(bw["nx"], 2, np.int32)
    shots = [1122 + 12 * i for i in range(S)]
    # plain: one shot of the same model
    with ttifd.Modeling(device=local_rank, **cfg) as h:
        h.upload_model(*pads)
        h.set_source([shots[0]], [2], wav)
        for k in (0, 1):
            h.set_receivers(k, gx, gz)
        h.reset()
        h.step(W)
        h.step(K)
        plain_ms = h.elapsed_ms
        cells = h.Nz * h.Nx
    plain = cells * K / (plain_ms / 1e3) / 1e9
    with ttifd.Batch([cfg], [0] * S, device=local_rank) as b:
        b.upload_model(0, *pads)
        for i, sx in enumerate(shots):
            inst = b.instances[i]
            inst.set_source([sx], [2], wav)
            for k in (0, 1):
                inst.set_receivers(k, gx, gz)
        tuned = b.autotune(min(20, K))
        b.reset()
        b.step(W)
        l0 = b.kernel_launches
        with ClockSampler(local_rank) as clk:
            b.step(K)
            ms = b.elapsed_ms
        launches = b.kernel_launches - l0
    value = S * cells * K / (ms / 1e3) / 1e9
    peak, src = peaks()
    state = 64 if variant == "tensor_rotation" else 40
    param = ALG_BYTES_STEP[variant] - state
    alg = (S * state + param) * cells * K / (ms / 1e3) / 1e9
    return {"workload": f"batched forward, {variant}, {S} shots 120 m apart on the 1126x3000 crop of the "
                        "salt-like model, 3000 receivers per shot, 10 Hz, ealThick=50, freesurface",
            "shots": S, "steps": K, "value": value, "unit": "Gcell/s", "ms_per_step": ms / K,
            "plain_same_model": plain, "speedup_vs_plain": value / plain,
            "schedule": tuned, "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": alg, "peak": peak, "unit": "GB/s", "frac": alg / peak,
                         "peak_source": src,
                         "alg_bytes_per_step": f"shots x cells x {state} B state + cells x {param} B parameters"},
            "clocks": clk.summary()}


def run_batched_uneven(args, local_rank):
    """Many independent models of different sizes in one batch (one launch per
    half-step over all of them): `uneven_models` layered models with seeded
    nz in [256, 1126], nx in [256, 4096], nt in [1000, 4000] (seed 4), one
    centred surface shot each, ealThick=40, receivers on every column at z=2.
    `batch_steps` steps are timed (instances whose nt is reached stay idle)."""
    import ttifd

    rng = np.random.default_rng(4)
    M, K, W = args.uneven_models, args.batch_steps, args.warmup
    sizes = [(int(rng.integers(256, 1127)), int(rng.integers(256, 4097)), int(rng.integers(1000, 4001)))
             for _ in range(M)]
    cfgs = [dict(variant=args.variant, nz=nz, nx=nx, nt=nt, dx=10.0, dz=10.0, dt=0.0008, fpeak=15.0, ealThick=40,
                 freesurface=0, stype=1, seistype=1, mt=1) for nz, nx, nt in sizes]
    with ttifd.Batch(cfgs, list(range(M)), device=local_rank) as b:
        cells = []
        for m, (nz, nx, nt) in enumerate(sizes):
            mod = synthetic.layered_model(nz, nx, seed=100 + m)
            b.upload_model(m, *synthetic.padded(mod, 40))
            inst = b.instances[m]
            inst.set_source([nx // 2], [2], synthetic.ricker(nt, 0.0008, 15.0)[None, :])
            for k in (0, 1):
                inst.set_receivers(k, np.arange(nx, dtype=np.int32), 2)
            cells.append(inst.Nz * inst.Nx)
        tuned = b.autotune(10)
        b.reset()
        b.step(W)
        with ClockSampler(local_rank) as clk:
            b.step(K)
            ms = b.elapsed_ms
        used = device_memory_in_use(local_rank)
    total = sum(cells)
    per = [c * K / (ms / 1e3) / 1e9 for c in cells]
    return {"workload": f"batched forward, {args.variant}, {M} independent layered models of seeded sizes "
                        "nz 256-1126, nx 256-4096, nt 1000-4000, one centred shot each, ealThick=40",
            "models": M, "steps": K, "cells_total": total, "value": total * K / (ms / 1e3) / 1e9, "unit": "Gcell/s",
            "ms_per_step": ms / K, "per_instance_gcells": {"min": min(per), "median": float(np.median(per)),
                                                            "max": max(per)},
            "window": f"rates over a window of {K} steps after {W} warm-up steps, not over each instance's whole "
                      "nt (every instance's nt is at least 1000, so all of them run through the window)",
            "device_memory_in_use_GB": used, "schedule": tuned, "clocks": clk.summary()}


def device_memory_in_use(device: int) -> float:
    """Device memory in use (total - free, GB) while the batch's buffers are held:
    the footprint of the run (this process's allocations, no other user)."""
    import torch

    free, total = torch.cuda.mem_get_info(device)
    return (total - free) / 1e9


# ---------------------------------------------------------------- gradient arm
GRAD_WORKLOAD = dict(nz=600, nx=1200, dx=10.0, dz=10.0, dt=0.0008, fpeak=12.0, ealThick=40, freesurface=0, stype=1,
                     seistype=1, mt=1, wsave=0, savew=0, mode=1, scalar=1.0, energy=0)


def run_gradient(args, local_rank):
    """One shot of the adjoint-state gradient (forward with checkpoints,
    recomputation, adjoint) against the plain forward of the same shot.
    True model: the layered generator at nz=600 nx=1200 (seed 3); start
    model: Gaussian blur (sigma 15 cells) of vp, epsilon, delta, theta, vs and
    rho derived from the blurred vp; surface shot at the centre, receivers at
    every x on z=5; `grad_steps` time steps with `grad_ncheck` checkpoints."""
    from scipy.ndimage import gaussian_filter

    import ttifd

    K, ncheck = args.grad_steps, args.grad_ncheck
    gw = dict(GRAD_WORKLOAD)
    true = synthetic.layered_model(gw["nz"], gw["nx"], seed=3)
    blur = [gaussian_filter(np.asarray(a, np.float64), 15.0).astype(np.float32)
            for a in (true.vp, true.epsilon, true.delta, true.theta)]
    vs = (blur[0] / 1.8).astype(np.float32)
    rho = (310.0 * blur[0] ** 0.25).astype(np.float32)
    start = synthetic.Model(blur[0], vs, rho, blur[1], blur[2], blur[3])
    true = synthetic.Model(true.vp, vs, rho, true.epsilon, true.delta, true.theta)
    cfg = dict(gw, variant="coordinate_rotation", nt=K)
    wav = synthetic.ricker(K, cfg["dt"], cfg["fpeak"])[None, :]
    gx = np.arange(gw["nx"], dtype=np.int32)
    with ttifd.Modeling(device=local_rank, **cfg) as h:
        h.upload_model(*synthetic.padded(true, gw["ealThick"]))
        h.set_source([gw["nx"] // 2], [2], wav)
        for k in (0, 1):
            h.set_receivers(k, gx, 5)
        h.run()
        dobs = [h.fetch_traces(k) for k in (0, 1)]
    with ttifd.Modeling(device=local_rank, **cfg) as h:
        h.upload_model(*synthetic.padded(start, gw["ealThick"]))
        h.set_source([gw["nx"] // 2], [2], wav)
        for k in (0, 1):
            h.set_receivers(k, gx, 5)
            h.grad_set_observed(k, dobs[k])
        h.reset()
        h.step(K)
        fwd_ms = h.elapsed_ms
        h.grad_zero()
        h.grad_run(ncheck)  # warm-up (allocations)
        h.grad_zero()
        J = h.grad_run(ncheck)
        grad_ms = h.elapsed_ms
        h.grad_zero()
        h.grad_run(30)  # the 30-checkpoint schedule: 29 segments recomputed
        grad30_ms = h.elapsed_ms
        cells = h.Nz * h.Nx
        gvp = h.grad_fetch("vp").astype(np.float64)  # values near 1e-20: norm in double
        gnorm, gmax = float(np.linalg.norm(gvp)), float(np.abs(gvp).max())
    return {"workload": f"adjoint-state gradient, coordinate_rotation, one surface shot on the layered 600x1200 "
                        f"model (padded {h.Nz}x{h.Nx}), blurred start model, {K} steps, {ncheck} checkpoints",
            "steps": K, "ncheck": ncheck, "forward_ms": fwd_ms, "gradient_ms": grad_ms,
            "cost_vs_forward": grad_ms / fwd_ms, "value": cells * K / (grad_ms / 1e3) / 1e9, "unit": "Gcell/s",
            "ncheck30_ms": grad30_ms, "ncheck30_cost_vs_forward": grad30_ms / fwd_ms,
            "misfit": J, "grad_vp_norm": gnorm, "grad_vp_max_abs": gmax}


def grad_models():
    """The gradient workload's true and start models (layered 600 x 1200, seed 3;
    start = Gaussian blur, sigma 15 cells = 150 m, of vp, epsilon, delta and theta;
    vs and rho derived from the blurred vp and held fixed)."""
    from scipy.ndimage import gaussian_filter

    gw = GRAD_WORKLOAD
    true = synthetic.layered_model(gw["nz"], gw["nx"], seed=3)
    blur = [gaussian_filter(np.asarray(a, np.float64), 15.0).astype(np.float32)
            for a in (true.vp, true.epsilon, true.delta, true.theta)]
    vs = (blur[0] / 1.8).astype(np.float32)
    rho = (310.0 * blur[0] ** 0.25).astype(np.float32)
    start = synthetic.Model(blur[0], vs, rho, blur[1], blur[2], blur[3])
    true = synthetic.Model(true.vp, vs, rho, true.epsilon, true.delta, true.theta)
    return true, start


def run_gradient_shots(args, local_rank):
    """The gradient configuration as specified: 16 surface shots evenly spaced
    on the 600 x 1200 layered model, `grad_steps` steps, 30 checkpoints (29
    full-state slots and a kept segment of steps / 30 steps, the states at the
    other segment starts recomputed), through tti_batch_grad_run (the shots'
    gradients at once, one stream each, parameters shared). Its cost is set
    against the batched forward of the same 16 shots (tti_batch_step,
    autotuned) and against 16 plain forwards."""
    import ttifd

    K, S = args.grad_steps, args.grad_shots
    gw = dict(GRAD_WORKLOAD)
    true, start = grad_models()
    cfg = dict(gw, variant="coordinate_rotation", nt=K)
    wav = synthetic.ricker(K, cfg["dt"], cfg["fpeak"])[None, :]
    gx = np.arange(gw["nx"], dtype=np.int32)
    shots = [int(round((i + 0.5) * gw["nx"] / S)) for i in range(S)]
    # observed traces: the true model's, all shots in one batch
    with ttifd.Batch([cfg], [0] * S, device=local_rank) as b:
        b.upload_model(0, *synthetic.padded(true, gw["ealThick"]))
        for i, sx in enumerate(shots):
            b.instances[i].set_source([sx], [2], wav)
            for k in (0, 1):
                b.instances[i].set_receivers(k, gx, 5)
        b.run()
        dobs = [[b.instances[i].fetch_traces(k) for k in (0, 1)] for i in range(S)]
    seg = -(-K // 30)
    with ttifd.Batch([cfg], [0] * S, device=local_rank) as b:
        b.upload_model(0, *synthetic.padded(start, gw["ealThick"]))
        for i, sx in enumerate(shots):
            inst = b.instances[i]
            inst.set_source([sx], [2], wav)
            for k in (0, 1):
                inst.set_receivers(k, gx, 5)
                inst.grad_set_observed(k, dobs[i][k])
        cells = b.instances[0].Nz * b.instances[0].Nx
        tuned = b.autotune(min(20, K))
        b.reset()
        b.step(K)
        fwd_ms = b.elapsed_ms
        b.grad_run(29, seg)  # warm-up: allocations, kernel attributes
        with ClockSampler(local_rank) as clk:
            Js = b.grad_run(29, seg)
            grad_ms = b.elapsed_ms
        used = device_memory_in_use(local_rank)
    with ttifd.Modeling(device=local_rank, **cfg) as h:  # one plain shot, for the sequential baseline
        h.upload_model(*synthetic.padded(start, gw["ealThick"]))
        h.set_source([shots[0]], [2], wav)
        h.reset()
        h.step(K)
        plain_ms = h.elapsed_ms
    return {"workload": f"adjoint-state gradient, coordinate_rotation, {S} surface shots on the layered 600x1200 "
                        f"model, blurred start model, {K} steps, 30 checkpoints (29 slots + a kept segment of "
                        f"{seg} steps)",
            "shots": S, "steps": K, "checkpoints": 30, "gradient_ms": grad_ms,
            "batched_forward_ms": fwd_ms, "cost_vs_batched_forward": grad_ms / fwd_ms,
            "plain_forward_ms_x_shots": plain_ms * S, "cost_vs_plain_forwards": grad_ms / (plain_ms * S),
            "value": S * cells * K / (grad_ms / 1e3) / 1e9, "unit": "Gcell/s (forward cell-updates of all shots "
                                                                   "per second of gradient)",
            "misfit_sum": float(sum(Js)), "device_memory_in_use_GB": used, "forward_schedule": tuned,
            "clocks": clk.summary()}


def run_gradient_full(args, local_rank):
    """The batched gradient on the full model: `grad_full_shots` shots 120 m
    apart around the surface centre of the 1126 x 7872 salt-like model
    (ealThick 60, free surface, 7872 receivers at z=2, observed traces zero so
    J = 1/2 |d|^2), `grad_full_steps` steps, checkpoints planned by
    tti_grad_plan for an equal share per shot of 90 % of the free device
    memory (less each shot's fixed buffers). The plan for the full nt = 5000
    under the same budget is reported beside it."""
    import ttifd

    S, K = args.grad_full_shots, args.grad_full_steps
    cfg = dict(WORKLOAD, variant="coordinate_rotation", nt=K, seistype=1, wsave=0, energy=0)
    m = model()
    pads = synthetic.padded(m, WORKLOAD["ealThick"])
    wav = synthetic.ricker(K, cfg["dt"], cfg["fpeak"])[None, :]
    nx = WORKLOAD["nx"]
    gx = np.arange(nx, dtype=np.int32)
    shots = [nx // 2 + 12 * (i - S // 2) for i in range(S)]
    with ttifd.Batch([cfg], [0] * S, device=local_rank) as b:
        b.upload_model(0, *pads)
        for i, sx in enumerate(shots):
            inst = b.instances[i]
            inst.set_source([sx], [2], wav)
            for k in (0, 1):
                inst.set_receivers(k, gx, 2)
                inst.grad_set_observed(k, np.zeros((nx, inst.nts), np.float32))
        cells = b.instances[0].Nz * b.instances[0].Nx
        tuned = b.autotune(min(20, K))
        b.reset()
        b.step(K)
        fwd_ms = b.elapsed_ms
        import torch

        free0, total = torch.cuda.mem_get_info(local_rank)
        n = b.instances[0].Nx * ((b.instances[0].Nz + 31) // 32 * 32)
        fixed = 4.0 * n * 27 + 4.0 * nx * K * 6  # adjoint fields and sums, traces, observed, residuals
        budget = max(0.0, (0.9 * free0) / S - fixed)
        plan = b.instances[0].grad_plan(budget)
        b.grad_run(plan["snapshots"], plan["keep_steps"])
        grad_ms = b.elapsed_ms
        used = device_memory_in_use(local_rank)
    try:
        with ttifd.Modeling(device=local_rank, **dict(cfg, nt=5000)) as h:
            plan5000 = h.grad_plan(budget)
    except ttifd.TTIError as e:
        plan5000 = {"error": str(e)}
    return {"workload": f"batched adjoint-state gradient, coordinate_rotation, {S} shots on the full 1126x7872 "
                        f"salt-like model (padded 1256x8002), {K} steps, checkpoints planned for a "
                        f"{budget / 1e9:.2f} GB share per shot",
            "shots": S, "steps": K, "gradient_ms": grad_ms, "batched_forward_ms": fwd_ms,
            "cost_vs_batched_forward": grad_ms / fwd_ms,
            "value": S * cells * K / (grad_ms / 1e3) / 1e9, "per_shot_gcells": cells * K / (grad_ms / 1e3) / 1e9,
            "unit": "Gcell/s", "plan": plan, "plan_nt5000_same_budget": plan5000,
            "device_memory_in_use_GB": used, "device_memory_total_GB": total / 1e9, "forward_schedule": tuned}


# ---------------------------------------------------------------- reference arm
def ref_program(variant: str):
    for sub in ("bin", "strict"):
        p = os.path.join(ROOT, "oracle", "_ref", sub, f"sufdmod2dTTIelastic_{variant}")
        if os.path.exists(p):
            return p, sub
    return None, None


def run_reference_cpu(variant: str, budget_s: float = 20.0, max_steps: int = 400):
    """Times the reference's own OpenMP build on this host's cores on the bench
    workload for a bounded number of steps; returns a cpu_baseline dict."""
    prog, build = ref_program(variant)
    if prog is None:
        return None
    m = model()
    work = tempfile.mkdtemp(prefix="ttifd_ref_")
    try:
        files = synthetic.write_model(work, m)
        sx, sz, gx, gz = geometry(0)
        ncores = os.cpu_count() or 1
        env = dict(os.environ, OMP_NUM_THREADS=str(ncores), OMP_PROC_BIND="close", OMP_PLACES="cores",
                   SUSHIM_QUIET="1")

        def once(nt):
            wav = synthetic.ricker(nt, WORKLOAD["dt"], WORKLOAD["fpeak"])
            synthetic.write_su_source(os.path.join(work, "src.su"), wav[None, :], [sx], [sz], WORKLOAD["dt"])
            synthetic.write_su_receivers(os.path.join(work, "rec.su"), gx, gz)
            # the same getpar values as our arm's workload (snapshots every
            # snap_sample steps written by the reference inside its timed loop)
            a = [f"{k}={v}" for k, v in WORKLOAD.items()] + [
                f"nt={nt}", "shotID=1", f"sourcefile={work}/src.su", f"recposfile={work}/rec.su"]
            a += [f"{k}file={files[k]}" for k in ("vp", "vs", "rho", "epsilon", "delta", "theta")]
            r = subprocess.run([prog] + a, cwd=work, env=env, capture_output=True, text=True)
            mt = re.search(r"Finite difference modeling takes ([0-9.eE+-]+) s", r.stdout)
            if r.returncode != 0 or not mt:
                raise RuntimeError(f"reference run failed ({r.returncode}): {r.stderr[-500:]}")
            return float(mt.group(1))

        t = once(10)
        steps = int(max(10, min(max_steps, 10 * budget_s / max(t, 1e-3))))
        t = once(steps)
        E = WORKLOAD["ealThick"] + 5
        cells = (WORKLOAD["nz"] + 2 * E) * (WORKLOAD["nx"] + 2 * E)
        return {"value": cells * steps / t / 1e9, "unit": "Gcell/s", "cores": ncores, "kind": "reference",
                "sample": f"{steps} steps of the same workload ({variant}), reference OpenMP build ({build}), "
                          f"loop time from its own 'Finite difference modeling takes' line: {t:.2f} s",
                "steps": steps, "loop_s": t}
    finally:
        shutil.rmtree(work, ignore_errors=True)


# ---------------------------------------------------------------- distributed
_G = None  # shots.Group


def dist_init():
    global _G
    import shots

    _G = shots.Group(timeout_s=300)
    return _G.rank, _G.world, _G.local_rank


def dist_barrier():
    _G.barrier()


def dist_max(x: float) -> float:
    return _G.max(x)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--variant", default="coordinate_rotation",
                    choices=["coordinate_rotation", "tensor_rotation", "bond_transformation"])
    ap.add_argument("--profile-steps", type=int, default=50)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--nx", type=int, default=WORKLOAD["nx"],
                    help="narrower model for profiler captures (default: the full 7872)")
    ap.add_argument("--batch-shots", type=int, default=64)
    ap.add_argument("--batch-steps", type=int, default=200)
    ap.add_argument("--no-batch", action="store_true", help="skip the batched measurement")
    ap.add_argument("--uneven-models", type=int, default=48)
    ap.add_argument("--grad-steps", type=int, default=3000)
    ap.add_argument("--grad-ncheck", type=int, default=1,
                    help="gradient segments (1: every state kept, as the 600x1200 case fits in HBM)")
    ap.add_argument("--no-grad", action="store_true", help="skip the gradient measurement")
    ap.add_argument("--grad-shots", type=int, default=16)
    ap.add_argument("--grad-full-shots", type=int, default=32)
    ap.add_argument("--grad-full-steps", type=int, default=200)
    ap.add_argument("--no-variants", action="store_true",
                    help="skip the other two formulations on the same workload")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    WORKLOAD["nx"] = args.nx
    rank, world, local_rank = dist_init()

    if args.impl == "reference":
        if rank == 0:
            cb = run_reference_cpu(args.variant)
            if cb is None:
                print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built on this host"}))
            else:
                line = {"impl": "reference", "metric": "Gcell-updates/s", "value": cb["value"], "unit": "Gcell/s",
                        "n_gpus": world, "steps": cb["steps"], "warmup": 0, "higher_is_better": True,
                        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                        "config": workload_config(args.variant, world),
                        "cpu_baseline": cb,
                        "e2e": {"value": cb["value"], "unit": "Gcell/s", "h2d_bytes_per_step": 0,
                                "d2h_bytes_per_step": 0}}
                print(json.dumps(line), flush=True)
        _G.close()
        return

    line = run_ours(args, rank, world, local_rank)
    if not args.no_batch and world == 1:
        line["batched"] = run_batched(args, local_rank)
        line["batched_uneven"] = run_batched_uneven(args, local_rank)
    if not args.no_grad and world == 1:
        line["gradient"] = run_gradient(args, local_rank)
        if args.grad_shots > 0:
            line["gradient_shots"] = run_gradient_shots(args, local_rank)
        if args.grad_full_shots > 0:
            line["gradient_batched_full"] = run_gradient_full(args, local_rank)
    if rank == 0:
        if not args.no_cpu_baseline:
            try:
                line["cpu_baseline"] = run_reference_cpu(args.variant)
            except Exception as e:  # reported, not fatal
                line["cpu_baseline"] = {"error": str(e)[:300]}
        print(json.dumps(line), flush=True)
    _G.close()


if __name__ == "__main__":
    main()
