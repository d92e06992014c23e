#!/usr/bin/env python
"""Benchmark of the MantlePar ML-WENO H/C transport + eutectic phase hot path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl mantlepar_b200|reference]

Metric: cell-updates/s (one cell advanced one accepted SSP-RK time step, all
stages). Workload (N=1): the plain FP64 single large instance, 1280x2560 uniform
quads on [0,0.5]x[0,1], seeded synthetic H/C/psi/Darcy data, SSPRK3 at CFL 0.4
(the reference integrates with SSPRK2; both are built). A bench step is one
accepted time step. The per-stage working set (~1.1 GB) exceeds the 126 MB L2,
so no flush is needed between steps.

value      device-timed (CUDA events) throughput with state resident in HBM;
e2e        the same metric through the C ABI with host buffers: per step the
           face velocities and H/C go host->device from pinned memory, the step
           runs, and H/C/T/phi come back device->host; the copies of the next
           step's inputs and the last step's results run on two copy streams
           during the current step (the sequential figure is reported beside);
roofline   one stage evaluation (the four stage kernels) counted as one launch
           against the measured HBM copy bandwidth (algorithmic 224 B/cell/stage),
           plus roofline_fp64 against a measured FP64 FMA peak (the binding roof);
cpu_baseline  the reference's own phase/mlweno/core sources (oracle/_ref) or the
           restated oracle, all host threads, on a bounded 160x320 sample.
Under torchrun (N>1) every rank advances its own 1280x2560 instance (replicas;
the instances are independent) and the max time over ranks is used.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(nx=1280, ny=2560)
# Algorithmic bytes per cell per stage: read U^(k) and U^n (32), write
# U^(k+1) (16), write T, phi (16), and the flow supplier's normal solid and
# Darcy velocities at the 5 Gauss points of the cell's 2 owned edges (2 x 80;
# both are per-point inputs, sampled from the flow solution in the reference).
ALG_BYTES_PER_CELL_STAGE = 224
# Executed FP64 operations per cell per stage (DFMA counted as 2, DADD/DMUL
# as 1) of the stage kernels, from an ncu capture of a 640x1280 stage:
# reconstruction 2073, cell phase 1188, faces 1703, accumulation ~48
# (per-cell figures are size-independent).
FP64_FLOPS_PER_CELL_STAGE = 5012
# DRAM bytes per cell per stage of the four stage kernels from the same capture
# (640x1280 keeps every stage array above L2 size; traffic scales with cells).
DRAM_BYTES_PER_CELL_STAGE = 924
# B200 FP64 (vector and tensor) datasheet figure per GPU of an HGX B200
# (296 TFLOP/s for 8 GPUs); the driver measures no FP64 peak.
FP64_DATASHEET_TFLOPS = 37.0
CPU_SAMPLE = dict(nx=160, ny=320)
CPU_SECONDS = 12.0


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 20 ms.

    The sampler starts before the timed region and waits for its first
    sample; each line is timestamped on arrival, and `summary` keeps the
    samples that arrived between `mark_start` and `mark_end`.
    """

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []
        self.t0 = self.t1 = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            deadline = time.monotonic() + 5.0
            while not self.lines and time.monotonic() < deadline and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append((time.monotonic(), line.strip()))

    def mark_start(self):
        self.t0 = time.monotonic()

    def mark_end(self):
        self.t1 = time.monotonic()

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lo = self.t0 if self.t0 is not None else -float("inf")
        hi = (self.t1 + 0.025) if self.t1 is not None else float("inf")
        for ts, line in self.lines:
            if not (lo <= ts <= hi):
                continue
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def host_available_bytes():
    """MemAvailable of the host (bytes), or None where it cannot be read."""
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return None


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_run(nsteps_min: int, seconds: float, threads: int, sample: dict | None = None):
    """Reference CPU implementation on the bounded sample: returns (value, cores, kind, sample, steps, time)."""
    from oracle import pyoracle as po
    from mantlepar_b200 import synthetic as sy
    kind = "reference" if po.reference_available() else "port"
    lib = po.reference() if kind == "reference" else po.restated()
    w = sy.Workload(**(sample or CPU_SAMPLE))
    t = po.TransportOracle(sy.material_s(), w, lib=lib, integrator=3, threads=threads)
    vs, ud = sy.face_velocity(w)
    H, C = sy.initial_state(w)
    t.set_face_velocity(vs, ud)
    t.set_state(H, C)
    code, _ = t.step(1)                 # first RHS + one step (not timed)
    assert code == 0
    steps, t0 = 0, time.perf_counter()
    while steps < nsteps_min or time.perf_counter() - t0 < seconds:
        code, _ = t.step(1)
        assert code == 0
        steps += 1
        if steps >= max(nsteps_min, 1) and time.perf_counter() - t0 >= seconds:
            break
    el = time.perf_counter() - t0
    t.close()
    return w.cells * steps / el, threads, kind, f"{w.nx}x{w.ny} sub-instance of the same construction, {steps} SSPRK3 steps", steps, el


def cpu_form_baseline(form: str, seconds: float = 6.0, threads: int = 0) -> dict:
    """The reference build (oracle/_ref; else the restated oracle) on a bounded
    160x320 sample of a form's workload, all host threads: cell-updates/s."""
    import sys as _sys
    from oracle import pyoracle as po
    from mantlepar_b200 import synthetic as sy
    threads = threads or os.cpu_count() or 1
    kind = "reference" if po.reference_available() else "port"
    lib = po.reference() if kind == "reference" else po.restated()
    w = sy.Workload(**CPU_SAMPLE)
    if form in ("preheat", "preheat_perturbed"):
        _sys.path.insert(0, os.path.join(ROOT, "tests"))
        import preheat_cases as pc
        quad = dict(family=sy.MESH_PERTURBED, perturbation=0.2, mesh_seed=11) if form == "preheat_perturbed" else {}
        case = pc.PreheatCase(w, through=0.05, kappa=1e-4, thermal_type=(1, 1, 0, 0),
                              thermal_value=(0.9, 0.2, 0.0, 0.0), end=1e9, dt_initial=1e-4, dt_max=1e-4, **quad)
        t = pc.oracle_instance(case, lib)
        assert t.preheat_begin()[0] == 0
        steps, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < seconds:
            code, rows = t.preheat_advance(5)
            assert code == 0
            steps += len(rows)
        sample = f"{w.nx}x{w.ny}{' perturbed' if quad else ''} sub-instance, {steps} forward-Euler steps"
    else:
        t = po.TransportOracle(sy.material_s(), w, lib=lib, integrator=3, threads=threads, mesh_family=1,
                               perturbation=0.2, mesh_seed=11)
        xy = t.vertices()
        t.set_face_velocity(*sy.face_velocity_quads(w, xy))
        t.set_state(*sy.initial_state(w))
        assert t.step(1)[0] == 0
        steps, t0 = 0, time.perf_counter()
        while steps < 1 or time.perf_counter() - t0 < seconds:
            assert t.step(1)[0] == 0
            steps += 1
        sample = f"{w.nx}x{w.ny} perturbed sub-instance, {steps} SSPRK3 steps"
    el = time.perf_counter() - t0
    t.close()
    return {"value": w.cells * steps / el, "unit": "cell-updates/s", "cores": threads, "kind": kind, "sample": sample}


def run_reference(args, world, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    from oracle import pyoracle as po
    from mantlepar_b200 import synthetic as sy
    kind = "reference" if po.reference_available() else "port"
    lib = po.reference() if kind == "reference" else po.restated()
    w = sy.Workload(**CPU_SAMPLE)
    t = po.TransportOracle(sy.material_s(), w, lib=lib, integrator=3, threads=threads)
    vs, ud = sy.face_velocity(w)
    H, C = sy.initial_state(w)
    t.set_face_velocity(vs, ud)
    t.set_state(H, C)
    code, _ = t.step(args.warmup)
    assert code == 0
    t0 = time.perf_counter()
    code, reps = t.step(args.steps)
    el = time.perf_counter() - t0
    assert code == 0
    value = w.cells * args.steps / el
    line = {"impl": "reference", "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": el * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(config_block(),
                           cpu_sample=f"{w.nx}x{w.ny} sub-instance of the same construction per step; the per-cell "
                                      "rate is extrapolated to the named workload (same config in name only)"),
            "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": threads, "kind": kind,
                             "sample": f"{w.nx}x{w.ny} sub-instance per step (bounded sample of the 1280x2560 workload), SSPRK3"},
            "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def config_block():
    return {"workload": f"plain FP64 transport+phase, single {WORKLOAD['nx']}x{WORKLOAD['ny']} instance on [0,0.5]x[0,1], SSPRK3, CFL 0.4",
            "nx": WORKLOAD["nx"], "ny": WORKLOAD["ny"], "integrator": "SSPRK3", "cfl": 0.4,
            "material": "S (Te0=250K, Tm0=1250K, L=6e5, cp=1200, Xe=0.5, alpha0=0)",
            "l2": "inputs larger than L2 (per-stage working set ~1.1 GB > 126 MB)"}


def rel_errors(got, ref):
    """Per-cell |x-ref|/max(|ref|, 1e-3*max|ref|) (max, L2) and normwise error."""
    scale = np.maximum(np.abs(ref), 1e-3 * np.max(np.abs(ref)))
    e = np.abs(got - ref) / scale
    return {"max": float(np.max(e)), "l2": float(np.sqrt(np.mean(e * e))),
            "normwise": float(np.max(np.abs(got - ref)) / np.max(np.abs(ref)))}


def timed_steps(obj, steps, stream):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    out = obj.step(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), out


# Legacy dry preheat (src/couple/preheat.cpp) per cell-step: unlimited H
# reconstruction (read H, write 9 coefficients), edge fluxes (read both
# sides' coefficients and averages, 2 edges x 5 normal velocities, write 2
# fluxes), update (read H and 4 fluxes, write H): 8 + 72 + 72 + 8 + 80 + 16 +
# 8 + 16 + 8 bytes.
PREHEAT_BYTES_PER_CELL_STEP = 288


def preheat_form(steps, stream, nx=None, ny=None, perturbed=False):
    """The legacy dry preheat on the plain mesh (1280x2560), or on the
    perturbed-quadrilateral mesh (perturbation 0.2, seed 11) with per-cell
    tables: forward Euler with kappa = 1e-4 and wall temperatures, the
    synthetic Stokes flow plus an upward through-flow of 0.05 (inflow at the
    bottom wall); `steps` accepted steps, device-timed on the instance's
    stream."""
    import torch
    from mantlepar_b200 import synthetic as sy
    from mantlepar_b200.preheat import Preheat, PreheatConfig
    w = sy.Workload(nx=nx or WORKLOAD["nx"], ny=ny or WORKLOAD["ny"])
    xy = None
    if perturbed:
        xy = sy.quad_vertices(w, sy.MESH_PERTURBED, 0.2, 11)
        vs, ud = sy.face_velocity_quads(w, xy)
        vs = vs + 0.05 * (ud / w.darcy)
    else:
        vs, _ = sy.face_velocity(w)
        vs = vs.copy()
        vs[:w.nx * (w.ny + 1)] -= 0.05
    H, Cc = sy.initial_state(w)
    p = Preheat(w, PreheatConfig(end=1e9, max_steps=1 << 40, dt_initial=1e-4, dt_max=1e-4, cfl=0.5,
                                 diffusivity=1e-4, thermal_type=(1, 1, 0, 0), thermal_value=(0.9, 0.2, 0.0, 0.0)),
                stream=stream.cuda_stream, vertices=xy)
    p.set_velocity(vs)
    p.set_state(H, Cc)
    _, limit, _ = p.begin()
    p.advance(3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    code, rows = p.advance(steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    p.close()
    ms_step = ms / steps
    nbytes = PREHEAT_BYTES_PER_CELL_STEP + (PREHEAT_QUAD_EXTRA_BYTES if perturbed else 0)
    return {"value": w.cells * steps / (ms * 1e-3), "unit": "cell-updates/s", "steps": steps,
            "ms_per_step": ms_step, "status": code, "accepted": len(rows),
            "max_balance_error": max(abs(r["balanceError"]) for r in rows),
            "achieved_gbs": nbytes * w.cells / (ms_step * 1e-3) / 1e9,
            "hbm_frac_of_measured": nbytes * w.cells / (ms_step * 1e-3) / 1e9 / peaks()[0],
            "bytes_per_cell_step": nbytes,
            "config": f"{w.nx}x{w.ny}{' perturbed (0.2, seed 11)' if perturbed else ''}, kappa=1e-4, wall "
                      f"temperatures bottom 0.9 / top 0.2, through-flow 0.05, dt = min(1e-4, rate limit {limit:.3g}), "
                      f"host round trip every 512 steps"}


# Per-cell tables a stage of the general-quad path streams (G0 72, S9 36,
# T4 48, S4 24, geometry 4 doubles).
QUAD_TABLE_BYTES_PER_CELL = 184 * 8
# What a preheat step on a general quad mesh reads beyond the uniform one:
# the per-cell tables, the normal-line spacing of the 2 owned edges x 5
# points, and one vertex (x, y) per cell.
PREHEAT_QUAD_EXTRA_BYTES = QUAD_TABLE_BYTES_PER_CELL + 2 * 5 * 8 + 16


def quads_form(steps, stream, nx=None, ny=None):
    """The plain FP64 workload on the reference's perturbed-quadrilateral mesh
    (perturbation 0.2, seed 11): per-cell tables in HBM, every evaluation
    point mapped from the cell corners; SSPRK3, device-timed steps."""
    import torch
    from mantlepar_b200 import synthetic as sy
    from mantlepar_b200.transport import Transport, TransportConfig
    w = sy.Workload(nx=nx or WORKLOAD["nx"], ny=ny or WORKLOAD["ny"])
    xy = sy.quad_vertices(w, sy.MESH_PERTURBED, 0.2, 11)
    t0 = time.perf_counter()
    t = Transport(w, TransportConfig(cfl=w.cfl, integrator=3), stream=stream.cuda_stream, vertices=xy)
    setup_s = time.perf_counter() - t0
    t.set_face_velocity(*sy.face_velocity_quads(w, xy))
    t.set_state(*sy.initial_state(w))
    t.step(1)
    t.profile(True)
    ms, (_, reps) = timed_steps(t, steps, stream)
    kms, kn = t.kernel_times()
    t.close()
    stages = 3 * steps + sum(r["retries"] for r in reps) * 3
    table_gbs = QUAD_TABLE_BYTES_PER_CELL * w.cells * kn[0] / max(kms[0], 1e-9) / 1e6
    return {"value": w.cells * steps / (ms * 1e-3), "unit": "cell-updates/s", "steps": steps, "ms_per_step": ms / steps,
            "retries": sum(r["retries"] for r in reps), "table_setup_s": setup_s,
            "tables_gbs_over_stage": table_gbs, "tables_frac_of_measured_hbm_over_stage": table_gbs / peaks()[0],
            "stage_kernels_ms": {"recon+cellphase+face": kms[0] / max(kn[0], 1), "sum": kms[3] / max(kn[3], 1)},
            "stages": stages,
            "config": f"{w.nx}x{w.ny} perturbed quadrilateral (0.2, seed 11), SSPRK3, CFL 0.4, material S"}


def run_forms(args, stream):
    """The mixed-precision large instance and the batched uneven meshes."""
    import torch
    from mantlepar_b200 import synthetic as sy
    from mantlepar_b200.batch import Batch
    from mantlepar_b200.transport import Transport, TransportConfig
    forms = {}
    # Mixed precision: 4096x4096, H noise 0.1, SSPRK3; errors against the FP64 path
    # (which matches the FP64 oracle to 1e-12 at the small sizes the oracle runs).
    w = sy.mixed_large()
    H, Cc = sy.initial_state(w)
    vs, ud = sy.face_velocity(w)
    res = {}
    for prec in (1, 0):
        t = Transport(w, TransportConfig(cfl=w.cfl, integrator=3, precision=prec), stream=stream.cuda_stream)
        t.set_face_velocity(vs, ud)
        t.set_state(H, Cc)
        ms, _ = timed_steps(t, args.mixed_steps, stream)
        res[prec] = (ms, t.get_state())
        t.close()
    errs = {name: rel_errors(a, b) for name, a, b in zip(["H", "C", "T", "phi"], res[1][1], res[0][1])}
    forms["mixed_4096x4096"] = {
        "value": w.cells * args.mixed_steps / (res[1][0] * 1e-3), "unit": "cell-updates/s",
        "fp64_value": w.cells * args.mixed_steps / (res[0][0] * 1e-3),
        "steps": args.mixed_steps, "errors_vs_fp64_path": errs,
        "bitwise_equal_to_fp64_path": all(bool(np.array_equal(a, b)) for a, b in zip(res[1][1], res[0][1])),
        "precision": "FP64 stage (the form's 1e-6 per-cell bar admits no FP32 value on this path; an exact "
                     "FP32 screen of the limiter scan measured slower than the FP64 scan)"}
    del res
    # Config 0: the 20x20 instance, 200 SSPRK3 steps, through the
    # single-instance path: device-resident steps (CUDA graph, one host wait
    # per 64 steps) and the host-driven loop (one host wait per stage).
    w0 = sy.plain_small()
    H0, C0 = sy.initial_state(w0)
    vs0, ud0 = sy.face_velocity(w0)
    small = {}
    for dev in (True, False):
        t = Transport(w0, TransportConfig(cfl=w0.cfl, integrator=3), stream=stream.cuda_stream)
        t.set_device_steps(dev)
        t.set_face_velocity(vs0, ud0)
        t.set_state(H0, C0)
        t.step(3)
        t.set_state(H0, C0)
        syncs0 = t.host_syncs()
        ms, (_, reps) = timed_steps(t, w0.steps, stream)
        small[dev] = (ms, t.host_syncs() - syncs0, sum(r["retries"] for r in reps), t.get_state())
        t.close()
    forms["plain_fp64_20x20"] = {
        "value": w0.cells * w0.steps / (small[True][0] * 1e-3), "unit": "cell-updates/s", "steps": w0.steps,
        "ms_per_step": small[True][0] / w0.steps, "host_syncs_per_step": small[True][1] / w0.steps,
        "retries": small[True][2],
        "host_loop": {"value": w0.cells * w0.steps / (small[False][0] * 1e-3), "ms_per_step": small[False][0] / w0.steps,
                      "host_syncs_per_step": small[False][1] / w0.steps},
        "device_equals_host_loop": all(bool(np.array_equal(a, b)) for a, b in zip(small[True][3], small[False][3])),
        "config": "20x20 on [0,0.5]x[0,1], SSPRK3, CFL 0.4, material S, single instance (state reset before timing)"}
    # The 20x20 case as an ensemble: 4096 independent 20x20 meshes (seeds
    # 0..4095) in one batch, 200 SSPRK3 steps, device-resident.
    ens = [sy.Workload(nx=20, ny=20, seed=k) for k in range(4096)]
    b = Batch(ens, TransportConfig(cfl=0.4, integrator=3), stream=stream.cuda_stream)
    for i, x in enumerate(ens):
        b.set_face_velocity(i, *sy.face_velocity(x))
        b.set_state(i, *sy.initial_state(x))
    b.step(1)
    # The C call directly with one report buffer: building 4096 x 200 report
    # records in Python would sit inside the timed window.
    from mantlepar_b200 import _capi
    rep_buf = (_capi.StepReport * (w0.steps * b.slots))()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    _capi.check(b._lib.mp_batch_step(b._h, w0.steps, rep_buf))
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    ok = all(b.info(i)["status"] == 0 and b.info(i)["accepted"] == w0.steps + 1 for i in range(len(ens)))
    b.close()
    ecells = sum(x.cells for x in ens)
    forms["batched_20x20_4096"] = {
        "value": ecells * w0.steps / (ms * 1e-3), "unit": "cell-updates/s", "instances": len(ens),
        "steps": w0.steps, "ms_per_step": ms / w0.steps, "all_instances_healthy": ok,
        "over_one_20x20": ecells * w0.steps / (ms * 1e-3) / forms["plain_fp64_20x20"]["value"],
        "config": "4096 independent 20x20 meshes (seeds 0..4095) in one batch, SSPRK3, CFL 0.4, device-resident"}
    # Batched: 256 uneven meshes (seed 3), 100 steps, mixed and FP64,
    # autotuned tiles, device-resident steps; FP64 also with the host loop.
    ws = sy.batched_instances(256, seed=3)
    cells = sum(x.cells for x in ws)
    nsteps = args.batch_steps
    for prec, name, dev in ((1, "batched_mixed_256", True), (0, "batched_fp64_256", True),
                            (0, "batched_fp64_256_host_loop", False)):
        b = Batch(ws, TransportConfig(cfl=0.4, integrator=3, precision=prec), stream=stream.cuda_stream)
        b.set_device_steps(dev)
        for i, x in enumerate(ws):
            vs_i, ud_i = sy.face_velocity(x)
            H_i, C_i = sy.initial_state(x)
            b.set_face_velocity(i, vs_i, ud_i)
            b.set_state(i, H_i, C_i)
        tile, _ = b.autotune(reps=1)
        b.step(1)
        syncs0 = b.host_syncs()
        ms, reps = timed_steps(b, nsteps, stream)
        ok = all(r[i]["status"] == 0 for r in reps for i in range(len(ws)))
        forms[name] = {"value": cells * nsteps / (ms * 1e-3), "unit": "cell-updates/s",
                       "instances": len(ws), "cells": cells, "steps": nsteps, "ms_per_step": ms / nsteps,
                       "host_syncs_per_step": (b.host_syncs() - syncs0) / nsteps,
                       "device_steps": dev, "autotuned_tile": list(tile), "all_instances_healthy": ok}
        b.close()
    # The same 256 meshes one at a time through the plain single-instance
    # FP64 path (device-resident steps): what running them without the
    # batched engine costs.
    ms_solo = 0.0
    for x in ws:
        t = Transport(x, TransportConfig(cfl=0.4, integrator=3), stream=stream.cuda_stream)
        t.set_face_velocity(*sy.face_velocity(x))
        t.set_state(*sy.initial_state(x))
        t.step(1)
        ms, _ = timed_steps(t, nsteps, stream)
        ms_solo += ms
        t.close()
    forms["plain_fp64_256_one_at_a_time"] = {
        "value": cells * nsteps / (ms_solo * 1e-3), "unit": "cell-updates/s", "instances": len(ws), "steps": nsteps,
        "note": "each of the 256 meshes advanced alone through mp_transport_step (device-resident steps), times summed"}
    # Batched general quad meshes: 64 of the uneven meshes as
    # perturbed-quadrilateral instances (perturbation 0.2), 20 SSPRK3 steps,
    # device-resident; and the same meshes one at a time.
    qws = sy.batched_instances(64, seed=3)
    qxy = [sy.quad_vertices(x, sy.MESH_PERTURBED, 0.2, 11 + k) for k, x in enumerate(qws)]
    qcells = sum(x.cells for x in qws)
    qsteps = 20
    b = Batch([], TransportConfig(cfl=0.4, integrator=3), stream=stream.cuda_stream)
    for x, xy in zip(qws, qxy):
        i = b.add_quads(x, xy)
        b.set_face_velocity(i, *sy.face_velocity_quads(x, xy))
        b.set_state(i, *sy.initial_state(x))
    b.step(1)
    ms, reps = timed_steps(b, qsteps, stream)
    ok = all(r[i]["status"] == 0 for r in reps for i in range(len(qws)))
    b.close()
    ms_solo = 0.0
    for x, xy in zip(qws, qxy):
        t = Transport(x, TransportConfig(cfl=0.4, integrator=3), stream=stream.cuda_stream, vertices=xy)
        t.set_face_velocity(*sy.face_velocity_quads(x, xy))
        t.set_state(*sy.initial_state(x))
        t.step(1)
        m1, _ = timed_steps(t, qsteps, stream)
        ms_solo += m1
        t.close()
    forms["batched_quads_64"] = {
        "value": qcells * qsteps / (ms * 1e-3), "unit": "cell-updates/s", "instances": len(qws), "cells": qcells,
        "steps": qsteps, "ms_per_step": ms / qsteps, "all_instances_healthy": ok,
        "one_at_a_time": {"value": qcells * qsteps / (ms_solo * 1e-3), "ms_per_step": ms_solo / qsteps},
        "config": "64 uneven meshes (nx 40..640, ny 40..960, seed 3) as perturbed-quadrilateral meshes (0.2), "
                  "SSPRK3, CFL 0.4, device-resident steps"}
    # Product-input features on the plain workload: thermal diffusion, a
    # lithostatic pressure and the adiabatic source (FP64).
    import dataclasses
    wp = sy.Workload(**WORKLOAD)
    mat = dataclasses.replace(sy.material_s(), rho=100.0, alpha0=3e-5)
    tp = Transport(wp, TransportConfig(material=mat, cfl=wp.cfl, integrator=3, diffusivity=1e-4),
                   stream=stream.cuda_stream)
    tp.set_thermal_bc((1, 1, 0, 0), (0.9, 0.2, 0.0, 0.0))
    tp.set_pressure_model(tp.LITHOSTATIC, 1.1)
    tp.set_cell_velocity(*sy.cell_velocity(wp))
    vs_p, ud_p = sy.face_velocity(wp)
    H_p, C_p = sy.initial_state(wp)
    tp.set_face_velocity(vs_p, ud_p)
    tp.set_state(H_p, C_p)
    tp.step(1)
    ms, (_, reps) = timed_steps(tp, args.form_steps, stream)
    forms["product_features_1280x2560"] = {
        "value": wp.cells * args.form_steps / (ms * 1e-3), "unit": "cell-updates/s", "steps": args.form_steps,
        "features": "kappa=1e-4 with wall temperatures, lithostatic pressure, adiabatic source (alpha0=3e-5)",
        "retries": sum(r["retries"] for r in reps)}
    tp.close()
    forms["preheat_1280x2560"] = preheat_form(max(args.form_steps, 50), stream)
    forms["preheat_perturbed_1280x2560"] = preheat_form(max(args.form_steps, 50), stream, perturbed=True)
    forms["perturbed_quads_1280x2560"] = quads_form(args.form_steps, stream)
    if not args.no_cpu_baseline:
        forms["preheat_1280x2560"]["cpu_baseline"] = cpu_form_baseline("preheat")
        forms["preheat_perturbed_1280x2560"]["cpu_baseline"] = cpu_form_baseline("preheat_perturbed")
        forms["perturbed_quads_1280x2560"]["cpu_baseline"] = cpu_form_baseline("quads")
    # Served (mixed precision, memory admission, continuous batching), two
    # runs of 200 requests of the seeded stream:
    #  (a) the specified load, 200 req/s with nx up to 1280: about 500 times
    #      one GPU's capacity, so the run is bounded in wall time and the
    #      requests still queued or running at the bound are reported as
    #      censored (their latency is at least the time they waited);
    #  (b) a load one GPU sustains: the same generator with nx up to 320,
    #      offered at 70% of the capacity measured in (a).
    if args.serve_requests > 0:
        from mantlepar_b200.serve import Server, input_bytes, poisson_requests, request_work, run_stream

        def served(reqs, wall, target):
            srv = Server(TransportConfig(cfl=0.4, integrator=3, precision=1), memory_budget=64 << 30)
            srv.set_policy(Server.SMALLEST_WORK, target)
            out = run_stream(srv, reqs, wall_limit=wall)
            srv.close()
            out.pop("results")
            return out

        reqs = poisson_requests(args.serve_requests, rate=200.0, seed=4)
        # Inputs are prepared before the clock (face velocities once per
        # mesh shape) and queued requests keep a copy in the server: keep
        # twice the inputs' bytes below a third of the host's free memory.
        avail = host_available_bytes()
        kept, total = [], 0
        for r in reqs:
            need = 2 * input_bytes(r)
            if avail and total + need > avail / 3:
                break
            kept.append(r)
            total += need
        reqs = kept
        # A backlog: the throughput setting of the resident-cell target.
        a = served(reqs, args.serve_wall, 4.0e6)
        forms["served_poisson_200rps"] = dict(
            a, requests_drawn=args.serve_requests, offered_rate_rps=200.0, arrival_span_s=reqs[-1].arrival,
            offered_cell_updates=float(sum(request_work(r) for r in reqs)),
            admission="smallest estimated work first, 4e6 resident cells, 64 GiB budget",
            note=f"nx in 20..1280; bounded at {args.serve_wall:.0f} s of wall time: completed requests give the "
                 "latency percentiles, censored ones are still queued or running")
        small = poisson_requests(args.serve_requests, rate=1.0, seed=5, max_nx=320)
        mean_work = float(np.mean([request_work(r) for r in small]))
        capacity = a["gpu_busy_value"] / mean_work
        rate = 0.7 * capacity
        small = poisson_requests(args.serve_requests, rate=rate, seed=5, max_nx=320)
        # A sustainable load: the server's default (latency) target.
        b_ = served(small, args.serve_wall, 1.0e6)
        forms["served_sustained"] = dict(
            b_, offered_rate_rps=rate, arrival_span_s=small[-1].arrival, capacity_rps_estimate=capacity,
            admission="smallest estimated work first, 1e6 resident cells (the default), 64 GiB budget",
            note="nx in 20..320 (ny = nx * U{1,2}, t_final U[0.01, 0.1]), offered at 70% of the capacity "
                 "estimated from run (a)'s GPU throughput and the stream's mean work")
    return forms


def run_gpu(args, world, rank, local):
    import torch
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
        pg = dist
    from mantlepar_b200 import _capi, synthetic as sy
    from mantlepar_b200.transport import Transport, TransportConfig
    import ctypes as C
    lib = _capi.lib()
    w = sy.Workload(**WORKLOAD, seed=1 + rank)
    stream = torch.cuda.current_stream(dev)
    t = Transport(w, TransportConfig(cfl=w.cfl, integrator=3), stream=stream.cuda_stream)
    vs, ud = sy.face_velocity(w)
    H, Cc = sy.initial_state(w)
    t.set_face_velocity(vs, ud)
    t.set_state(H, Cc)
    t.step(max(args.warmup, 1))

    def barrier():
        if pg:
            pg.barrier()
        torch.cuda.synchronize()

    # ---- resident throughput: the default device-resident steps (CUDA graph,
    # step decisions on the device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = _capi.kernel_launches()
    syncs0 = t.host_syncs()
    barrier()
    with ClockSampler(local) as clk:
        barrier()
        clk.mark_start()
        e0.record(stream)
        _, reps = t.step(args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        clk.mark_end()
    launches = _capi.kernel_launches() - launches0
    host_syncs = t.host_syncs() - syncs0
    ms = e0.elapsed_time(e1)
    # ---- per-kernel CUDA-event timing for the roofline: a second run of
    # the same length through the host-driven loop (events around every
    # kernel on the transport's stream)
    _capi.check(lib.mp_transport_profile(t._h, 1))
    e0p, e1p = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    e0p.record(stream)
    _, reps_p = t.step(args.steps)
    e1p.record(stream)
    torch.cuda.synchronize()
    ms_profiled = e0p.elapsed_time(e1p)
    kms = (C.c_double * 6)()
    kn = (C.c_ulonglong * 6)()
    _capi.check(lib.mp_transport_kernel_times(t._h, kms, kn))
    _capi.check(lib.mp_transport_profile(t._h, 0))
    ms_max = ms
    if pg:
        x = torch.tensor([ms], device=dev, dtype=torch.float64)
        pg.all_reduce(x, op=pg.ReduceOp.MAX)
        ms_max = float(x.item())
    cells = w.cells
    value = world * cells * args.steps / (ms_max * 1e-3)
    retries = sum(r["retries"] for r in reps)

    # ---- end to end through the C ABI with pinned host buffers
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    hv, hu, hH, hC = pin(vs), pin(ud), pin(H), pin(Cc)
    oH, oC, oT, oP = (torch.empty(cells, dtype=torch.float64).pin_memory() for _ in range(4))
    # (a) sequential: each call copies straight from / to the host buffers.
    barrier()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        t.set_face_velocity(hv, hu)
        t.set_state(hH, hC)
        t.step(1)
        t.get_state_into(oH, oC, oT, oP)
    e3.record(stream)
    torch.cuda.synchronize()
    ms_seq = e2.elapsed_time(e3)
    seq_out = [x.clone() for x in (oH, oC, oT, oP)]
    # (b) pipelined: step k+1's inputs go host->device on one copy stream
    # while step k runs, and step k's results go device->host on another
    # while step k+1 runs (the link carries both directions at once);
    # double-buffered device staging, the calls take the device buffers.
    c_in, c_out = torch.cuda.Stream(), torch.cuda.Stream()
    stage_in = [[torch.empty(x.numel(), dtype=torch.float64, device=dev) for x in (hv, hu, hH, hC)] for _ in range(2)]
    stage_out = [[torch.empty(cells, dtype=torch.float64, device=dev) for _ in range(4)] for _ in range(2)]
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_out = [torch.cuda.Event() for _ in range(2)]

    def upload(k):
        b = k & 1
        with torch.cuda.stream(c_in):
            for d, h in zip(stage_in[b], (hv, hu, hH, hC)):
                d.copy_(h.view(-1), non_blocking=True)
            ev_in[b].record(c_in)

    barrier()
    e4, e5 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e4.record(stream)
    c_in.wait_stream(stream)
    upload(0)
    for k in range(args.steps):
        b = k & 1
        if k + 1 < args.steps:
            upload(k + 1)        # the buffer of step k-1, whose synchronous set calls have returned
        stream.wait_event(ev_in[b])
        sv, su, sH, sC = stage_in[b]
        t.set_face_velocity(sv, su)
        t.set_state(sH, sC)
        t.step(1)
        if k >= 2:
            ev_out[b].synchronize()                     # step k-2's results have left this buffer
        t.get_state_into(*stage_out[b])
        c_out.wait_stream(stream)
        with torch.cuda.stream(c_out):
            for d, h in zip(stage_out[b], (oH, oC, oT, oP)):
                h.copy_(d, non_blocking=True)
            ev_out[b].record(c_out)
    stream.wait_stream(c_out)
    stream.wait_stream(c_in)
    e5.record(stream)
    torch.cuda.synchronize()
    ms_e2e = e4.elapsed_time(e5)
    # Every step restarts from the same inputs, so both loops end on the same result.
    pipe_same = all(bool(torch.equal(a, b)) for a, b in zip(seq_out, (oH, oC, oT, oP)))
    if pg:
        x = torch.tensor([ms_e2e, ms_seq], device=dev, dtype=torch.float64)
        pg.all_reduce(x, op=pg.ReduceOp.MAX)
        ms_e2e, ms_seq = float(x[0].item()), float(x[1].item())
    e2e_value = world * cells * args.steps / (ms_e2e * 1e-3)
    e2e_seq_value = world * cells * args.steps / (ms_seq * 1e-3)
    h2d = hv.numel() * 8 + hu.numel() * 8 + hH.numel() * 8 + hC.numel() * 8
    d2h = 4 * cells * 8

    # ---- roofline of one stage (reconstruction + cell phase + face + sum kernels)
    stages = kn[0]
    stage_ms = (kms[0] + kms[1] + kms[2] + kms[3]) / max(stages, 1)
    hbm_peak, peak_kind = peaks()
    achieved = ALG_BYTES_PER_CELL_STAGE * cells / (stage_ms * 1e-3) / 1e9
    traffic = DRAM_BYTES_PER_CELL_STAGE * cells if DRAM_BYTES_PER_CELL_STAGE else None
    fp64 = C.c_double(0)
    _capi.check(lib.mp_probe_fp64_peak(stream.cuda_stream, C.byref(fp64)))
    total_k = sum(kms[k] for k in range(5))
    names = ["recon", "cellphase", "face", "sum", "axpy_reduce"]
    shares = {n: round(kms[k] / total_k, 4) if total_k else None for k, n in enumerate(names)}
    kernel_ms = {n: kms[k] / max(kn[k], 1) for k, n in enumerate(names)}
    line = None
    if rank == 0:
        roof64 = {"bound": "fp64", "peak": fp64.value, "unit": "TFLOP/s", "peak_kind": "measured (FMA probe)",
                  "peak_datasheet": FP64_DATASHEET_TFLOPS}
        if FP64_FLOPS_PER_CELL_STAGE:
            a64 = FP64_FLOPS_PER_CELL_STAGE * cells / (stage_ms * 1e-3) / 1e12
            roof64.update(achieved=a64, frac=a64 / fp64.value, frac_of_datasheet=a64 / FP64_DATASHEET_TFLOPS,
                          flops_per_cell_stage=FP64_FLOPS_PER_CELL_STAGE)
        else:
            roof64.update(achieved=None, frac=None)
        line = {
            "metric": "cell-updates/s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config_block(),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak, "traffic": traffic,
                         "peak_kind": peak_kind + " copy bandwidth",
                         "kernel": "one stage = recon_kernel + cellphase_kernel + face_kernel + sum_kernel",
                         "stage_ms": stage_ms, "stages_timed": int(stages), "kernel_shares": shares,
                         "kernel_avg_ms": kernel_ms},
            "roofline_fp64": roof64,
            "e2e": {"value": e2e_value, "unit": "cell-updates/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": ms_e2e / args.steps,
                    "pipeline": "step k+1's inputs host->device and step k-1's results device->host on two copy "
                                "streams while step k runs (double-buffered device staging)",
                    "sequential": {"value": e2e_seq_value, "ms_per_step": ms_seq / args.steps},
                    "pipelined_equals_sequential": pipe_same},
            "gpu_launches": int(launches),
            "host_syncs_per_step": host_syncs / args.steps,
            # The host-driven loop's run continues from the timed run's end
            # state, so its steps take other retries: compare per stage.
            "host_loop_ms_per_step": ms_profiled / args.steps,
            "host_loop_retries": sum(r["retries"] for r in reps_p),
            "host_loop_ms_per_stage": ms_profiled / max(1, int(kn[0])),
            "clocks": clk.summary(),
            "retries": retries,
        }
    t.close()
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    if rank == 0 and world == 1 and not args.no_forms:
        forms = run_forms(args, torch.cuda.current_stream(dev))
        forms["plain_fp64_1280x2560"] = {"value": value, "unit": "cell-updates/s"}
        forms["batched_mixed_over_plain_fp64"] = forms["batched_mixed_256"]["value"] / value
        forms["batched_mixed_over_plain_fp64_same_meshes"] = (forms["batched_mixed_256"]["value"] /
                                                              forms["plain_fp64_256_one_at_a_time"]["value"])
        line["forms"] = forms
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, cores, kind, sample, _, _ = cpu_run(2, CPU_SECONDS, os.cpu_count() or 1)
        line["cpu_baseline"] = {"value": v, "unit": "cell-updates/s", "cores": cores, "kind": kind, "sample": sample}
        # The same sample on one core, recorded beside the all-core figure.
        v1, _, _, sample1, _, _ = cpu_run(1, CPU_SECONDS / 3, 1, dict(nx=40, ny=80))
        line["cpu_baseline"]["one_core"] = {"value": v1, "cores": 1, "sample": sample1}
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_decomposed(args, world, rank, local):
    """One mesh cut into `world` row slabs, one per GPU (strong scaling): halo
    rows over NCCL point-to-point, stage totals over NCCL all-reduce."""
    import datetime
    import torch
    import torch.distributed as dist
    from mantlepar_b200 import _capi, synthetic as sy
    from mantlepar_b200.domain import DistExchange, Slab, partition
    from mantlepar_b200.transport import TransportConfig
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    else:
        import socket
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        dist.init_process_group("nccl", store=dist.TCPStore("127.0.0.1", port, 1, True), rank=0, world_size=1,
                                device_id=dev)
    try:
        w = sy.Workload(**WORKLOAD)
        rows = partition(w.ny, world)
        slab = Slab(w, rows[rank], TransportConfig(cfl=w.cfl, integrator=3))
        vs, ud = sy.face_velocity(w)
        H, Cc = sy.initial_state(w)
        slab.set_face_velocity(vs, ud)
        slab.set_state(H, Cc)
        if world > 1:   # one slab is the whole mesh: nothing to exchange
            DistExchange(rank, world, rows, w.nx, device=dev).attach(slab)
        code, _ = slab.step(max(args.warmup, 1))
        _capi.check(code)
        dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(slab.stream)
        code, reps = slab.step(args.steps)
        e1.record(slab.stream)
        torch.cuda.synchronize()
        _capi.check(code)
        x = torch.tensor([e0.elapsed_time(e1)], device=dev, dtype=torch.float64)
        dist.all_reduce(x, op=dist.ReduceOp.MAX)
        ms = float(x.item())
        if rank == 0:
            line = {"metric": "cell-updates/s", "value": w.cells * args.steps / (ms * 1e-3), "unit": "cell-updates/s",
                    "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                    "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
                    "data": "synthetic",
                    "config": dict(config_block(), workload=f"plain FP64 transport+phase, one {w.nx}x{w.ny} instance "
                                                            f"in {world} row slabs (2-row halos over NCCL)",
                                   parallelism=f"row-slab domain decomposition x{world}"),
                    "retries": sum(r["retries"] for r in reps)}
            print(json.dumps(line), flush=True)
        slab.close()
    finally:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mantlepar_b200", choices=["mantlepar_b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-forms", action="store_true", help="skip the mixed / batched forms")
    ap.add_argument("--serve-requests", type=int, default=200)
    ap.add_argument("--serve-wall", type=float, default=90.0, help="wall-time bound of each served run (s)")
    ap.add_argument("--form-steps", type=int, default=5, help="timed steps of each extra form")
    ap.add_argument("--mixed-steps", type=int, default=50, help="steps of the mixed-precision 4096x4096 form")
    ap.add_argument("--batch-steps", type=int, default=100, help="steps of the 256-mesh batched forms")
    ap.add_argument("--nx", type=int, default=WORKLOAD["nx"], help="cells in x (profiling of smaller cases)")
    ap.add_argument("--ny", type=int, default=WORKLOAD["ny"], help="cells in y")
    ap.add_argument("--preheat-only", action="store_true",
                    help="time only the legacy dry preheat form (profiling)")
    ap.add_argument("--quads-only", action="store_true",
                    help="time only the perturbed-quadrilateral form (profiling)")
    ap.add_argument("--perturbed", action="store_true",
                    help="with --preheat-only: the preheat on the perturbed-quadrilateral mesh")
    ap.add_argument("--decompose", action="store_true",
                    help="one mesh in row slabs across the ranks (strong scaling) instead of one mesh per rank")
    args = ap.parse_args()
    WORKLOAD.update(nx=args.nx, ny=args.ny)
    world, rank, local = dist_setup()
    if args.preheat_only:
        import torch
        torch.cuda.set_device(local)
        print(json.dumps({"form": "preheat_perturbed" if args.perturbed else "preheat",
                          **preheat_form(args.steps, torch.cuda.Stream(), args.nx, args.ny, args.perturbed)}))
        return
    if args.quads_only:
        import torch
        torch.cuda.set_device(local)
        print(json.dumps({"form": "perturbed_quads", **quads_form(args.steps, torch.cuda.Stream(), args.nx, args.ny)}))
        return
    if args.impl == "reference":
        run_reference(args, world, rank)
    elif args.decompose:
        run_decomposed(args, world, rank, local)
    else:
        run_gpu(args, world, rank, local)


if __name__ == "__main__":
    main()
