"""Benchmark of the Roe-Exner SSPRK2 step on B200 (one JSON line on stdout, rank 0).

Workload (default): the Gaussian-bed Roe-Exner case, 2048 x 2048 cells (+ ring),
dx = 0.01 m, MPM bedload, Transmissive x / Reflective y, CFL 0.5, SSPRK2, float32 —
the configuration the metric is quoted on.  A step is one full SSPRK2 step (CFL
reduction + two fused stage kernels) over every physical cell; one cell advanced by one
step is one cell-update.

Reported:
  value      cell-updates/s of the device loop (graph replay), state resident in HBM,
             L2 flushed between timed steps and excluded from the timing (a 256 MiB write,
             then a 256 MiB read of another buffer, so that the timed step starts with
             no state in L2 and without the flush's dirty lines to write back);
  e2e        the same metric through the public API with host buffers: pinned-host ->
             device copy of the state, init, ``run_steps`` for all K steps, device -> host
             copy of the state, all inside the timed region (the second such call: the
             first, untimed, warms the allocator and captures the step graph);
  roofline   the stage kernels' algorithmic bytes per launch over their CUDA-event
             duration, against the measured HBM copy bandwidth;
  fp64       the same loop in float64 (the plain FP64 GPU path) and its speed ratio;
  accuracy   after 2000 SSPRK2 steps: rel-L1 and L-inf of h, hu, hv and z+z_b, float32
             vs float64 on the GPU at 2048^2 and both GPU precisions vs the float64 C
             oracle at 1024^2, with the volume-budget closure of each GPU run;
  cpu_baseline  the float32 build of the C/OpenMP restatement of the reference step (all
             host threads) on the 2048^2 workload itself, steps until about 10 s of CPU
             work;
  plain_roe  the plain Roe dam-break (256^2, float64, SSPRK2, 200 steps)
             and the NumPy oracle on the host for 10 steps of it;
  transport_case  the same case started at u = 1 m/s (Shields number about 0.15, bedload
             in every cell, so the stage kernel's sediment-free fast path never fires);
  ensemble   the ragged ensemble workload (64 Roe-Exner dam breaks, sides U{128..1024},
             own beds, step heights and dts; float32; 1000 SSPRK2 steps): autotuned band
             height, cell-updates/s over all members (state ~1.1 GB, larger than L2); under
             torchrun the members are split over the ranks and the rates summed;
  bandwidth_case  the same generator at 8192^2, K timed steps;
  adjoint    the configuration-4 inflow case (512^2, float64): forward and checkpointed
             backward ms per SSPRK2 step with the parameter adjoints.

``--impl reference`` times the reference algorithm on the CPU instead (the float32 build
of the C/OpenMP restatement of PyExner's JAX step, oracle/c, on the 2048^2 workload, the
float64 build timed beside it; JAX itself is not installed on these hosts) and prints its
line with "impl": "reference".
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

METRIC = "cell-updates/s Roe-Exner SSPRK2 FP32 vs FP64 at stated L1 err; % HBM peak"
UNIT = "cell-updates/s"
# algorithmic words per cell per launch of the stage / CFL kernels
WORDS_STAGE1 = 10   # reads h hu hv z_b z n_b, writes h hu hv z_b
WORDS_STAGE2 = 16   # reads h hu hv z_b z n_b + u^n h hu hv z_b G, writes h hu hv z_b G
WORDS_CFL = 4       # reads h hu hv G


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled while the timed region runs.

    Reads NVML in a host thread every 2 ms (read-only queries); falls back to
    ``nvidia-smi -lms 100`` when NVML is unavailable."""

    def __init__(self, index=0):
        self.index = index
        self.sm = []
        self.max = None
        self.reasons = set()
        self._stop = threading.Event()
        self._nvml = None
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.index)
            self.max = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            names = {pynvml.nvmlClocksEventReasonHwSlowdown: "hw_slowdown",
                     pynvml.nvmlClocksEventReasonHwThermalSlowdown: "hw_thermal_slowdown",
                     pynvml.nvmlClocksEventReasonSwThermalSlowdown: "sw_thermal_slowdown",
                     pynvml.nvmlClocksEventReasonSwPowerCap: "sw_power_cap"}

            def run():
                while not self._stop.is_set():
                    try:
                        self.sm.append(float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)))
                        r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                        for bit, nm in names.items():
                            if r & bit:
                                self.reasons.add(nm)
                    except Exception:
                        pass
                    time.sleep(0.002)

            self._nvml = pynvml
            self.t = threading.Thread(target=run, daemon=True)
            self.t.start()
        except Exception:
            self._start_smi()
        return self

    def _start_smi(self):
        q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=lambda: [self.lines.append(l.strip()) for l in self.proc.stdout],
                                      daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None

    def __exit__(self, *a):
        self._stop.set()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        elif self._nvml is not None:
            self.t.join(timeout=1)

    def summary(self):
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            parts = [p.strip() for p in l.split(",")]
            if len(parts) < 6:
                continue
            try:
                self.sm.append(float(parts[0]))
                self.max = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[2:6]):
                if v.lower().startswith("active"):
                    self.reasons.add(nm)
        return {"sm_mhz": statistics.median(self.sm) if self.sm else None, "sm_max_mhz": self.max,
                "reasons": sorted(self.reasons), "samples": len(self.sm)}


def max_over_ranks(sec, world, device):
    """The timed interval of the slowest rank (replicas: one all-reduce of the timing, no
    data-path collective)."""
    if world <= 1:
        return float(sec)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(sec)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t)


def sum_over_ranks(x, world, device):
    """Sum of a per-rank count (one all-reduce of a timing-side scalar)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t)


def replica_throughput(world, cells, steps, sec):
    """Whole-job cell-updates/s: every rank advances its own replica of ``cells`` cells."""
    return world * cells * steps / sec


def build_case(n, dtype, device, u0=0.1):
    import torch

    from pyexner_b200 import RoeExnerState, cases, create_solver_bundle

    c = cases.gaussian_bed(n, device=device, u0=u0)
    st = RoeExnerState.from_numpy(c["arrs"], c["seds"], dtype)
    bundle = create_solver_bundle("Roe Exner")
    cfg = bundle.config(st, None, c["boundaries"], c["dx"], c["params"])
    mask = bundle.mask_fn(st, None, c["boundaries"].boundary_mask)
    st = bundle.init_fn(st, mask, cfg)
    torch.cuda.synchronize()
    return c, bundle, cfg, mask, st


class L2Flush:
    """Untimed L2 flush between timed steps: write a 256 MiB buffer (larger than the
    126 MB L2), then read another 256 MiB one, which evicts the written lines, so the
    timed step neither finds its state in L2 nor pays for writing the flush back."""

    def __init__(self, device="cuda"):
        import torch

        n = 256 * 1024 * 1024 // 4
        self.w = torch.empty(n, dtype=torch.float32, device=device)
        self.r = torch.zeros(n, dtype=torch.float32, device=device)

    def zero_(self):
        self.w.zero_()
        self.r.sum()


def timed_device_loop(st, mask, cfg, steps, warmup, flush):
    """Graph-replayed SSPRK2 steps, one step per timed interval, L2 flushed between."""
    import torch

    from pyexner_b200 import run_steps
    from pyexner_b200.integrators import check_state, scratch_like

    b = scratch_like(st)
    run_steps(st, mask, cfg, "SSPRK2", warmup, 0.5, scratch=b)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    total = 0.0
    for _ in range(steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run_steps(st, mask, cfg, "SSPRK2", 1, 0.5, scratch=b, log_dt=False)
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1) / 1e3
    check_state(st, mask, cfg)
    return total, b


def kernel_breakdown(st, b, mask, cfg, steps, flush):
    """CUDA-event duration of each kernel (CFL, stage 1, stage 2) over ``steps`` steps."""
    import ctypes

    import torch

    from pyexner_b200 import _lib
    from pyexner_b200.solvers import _re_plan, _stream

    plan = _re_plan(st, mask, cfg)
    dt = torch.empty((), dtype=st.dtype, device=st.h.device)
    stream = torch.cuda.current_stream()
    A = st.c_fields()
    B1 = b.c_fields()
    B1.G = None
    B1.z = st.z.data_ptr()
    B1.n_b = st.n_b.data_ptr()
    B2 = b.c_fields()
    B2.z = st.z.data_ptr()
    B2.n_b = st.n_b.data_ptr()
    acc = {"cfl": 0.0, "stage1": 0.0, "stage2": 0.0}
    for _ in range(steps):
        flush.zero_()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        ev[0].record(stream)
        _lib.call("pxb_re_cfl", plan.handle, ctypes.byref(A), 0.5, ctypes.c_void_p(dt.data_ptr()), _stream())
        ev[1].record(stream)
        _lib.call("pxb_re_stage", plan.handle, ctypes.byref(A), ctypes.byref(B1), None,
                  ctypes.c_void_p(dt.data_ptr()), 0.0, _stream())
        ev[2].record(stream)
        _lib.call("pxb_re_stage", plan.handle, ctypes.byref(B2), ctypes.byref(A), ctypes.byref(A),
                  ctypes.c_void_p(dt.data_ptr()), 0.0, _stream())
        ev[3].record(stream)
        ev[3].synchronize()
        acc["cfl"] += ev[0].elapsed_time(ev[1]) / 1e3
        acc["stage1"] += ev[1].elapsed_time(ev[2]) / 1e3
        acc["stage2"] += ev[2].elapsed_time(ev[3]) / 1e3
    return {k: v / steps for k, v in acc.items()}


def e2e_run(n, dtype, steps, warmup):
    """Host buffers in, host buffers out, through the public API."""
    import torch

    from pyexner_b200 import RoeExnerState, cases, create_solver_bundle, run_steps

    c = cases.gaussian_bed(n, device="cuda")
    # the inputs of init_fn_roeexner in MPM mode: G is recomputed from h, hu, hv
    # (roe_exner_solver.py:58-78), so it is not copied in
    planes = ("h", "hu", "hv", "z", "z_b", "n")
    host = {k: torch.from_numpy(np.ascontiguousarray(c["arrs"][k])).to(dtype).pin_memory() for k in planes}
    out = {k: torch.empty_like(host["h"]).pin_memory() for k in ("h", "hu", "hv", "z_b", "G")}
    st = RoeExnerState.from_numpy(c["arrs"], c["seds"], dtype)
    bundle = create_solver_bundle("Roe Exner")
    cfg = bundle.config(st, None, c["boundaries"], c["dx"], c["params"])
    mask = bundle.mask_fn(st, None, c["boundaries"].boundary_mask)
    st = bundle.init_fn(st, mask, cfg)
    run_steps(st, mask, cfg, "SSPRK2", warmup, 0.5)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()

    def call():
        for k in planes:
            getattr(st, k).copy_(host[k], non_blocking=True)
        st2 = bundle.init_fn(st, mask, cfg)
        run_steps(st2, mask, cfg, "SSPRK2", steps, 0.5, log_dt=False)
        for k in out:
            out[k].copy_(getattr(st2, k), non_blocking=True)

    call()  # untimed: warms the allocator and captures the step graph for these buffers
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    call()
    e1.record(stream)
    e1.synchronize()
    sec = e0.elapsed_time(e1) / 1e3
    h2d = sum(v.numel() * v.element_size() for v in host.values())
    d2h = sum(v.numel() * v.element_size() for v in out.values())
    return sec, h2d, d2h


def gpu_run_with_budget(n, dtype, steps):
    """``steps`` SSPRK2 steps of the Gaussian-bed case at n x n on the GPU with the volume
    budget on; returns the final state and the budget closure (volume(end) - volume(start)
    + outflow, relative to the start volume, for water and sediment)."""
    import torch

    from pyexner_b200 import new_budget, outflow, run_steps, volume

    c, bundle, cfg, mask, st = build_case(n, dtype, "cuda")
    w0, z0 = volume(st, mask, cfg)
    bud = new_budget()
    run_steps(st, mask, cfg, "SSPRK2", steps, 0.5, budget=bud, log_dt=False)
    torch.cuda.synchronize()
    w1, z1 = volume(st, mask, cfg)
    ow, oz = outflow(bud)
    return st.to_numpy(), {"water_outflow_m3": ow, "sediment_outflow_m3": oz,
                           "water_closure_rel": (w1 - w0 + ow) / w0, "sediment_closure_rel": (z1 - z0 + oz) / z0}


def accuracy_run(n, steps, n_oracle, oracle_proc, oracle_path):
    """Float32 against float64 on the GPU at n x n after ``steps`` SSPRK2 steps, and at
    n_oracle x n_oracle both GPU precisions against the float64 C oracle (run by the
    spawned ``oracle_proc``), each with its volume-budget closure."""
    import torch

    res = {}
    for dt in (torch.float32, torch.float64):
        res[dt] = gpu_run_with_budget(n, dt, steps)
    out = {"steps": steps, "n": n, "fp32_vs_fp64_gpu": errors_vs(res[torch.float32][0], res[torch.float64][0]),
           "budget_fp32": res[torch.float32][1], "budget_fp64": res[torch.float64][1]}
    out["h_rel_l1"] = out["fp32_vs_fp64_gpu"]["h"]["rel_l1"]
    out["bed_rel_l1"] = out["fp32_vs_fp64_gpu"]["bed"]["rel_l1"]
    if oracle_proc is not None:
        g32, _ = gpu_run_with_budget(n_oracle, torch.float32, steps)
        g64, _ = gpu_run_with_budget(n_oracle, torch.float64, steps)
        oracle_proc.join()
        if oracle_proc.exitcode == 0 and os.path.exists(oracle_path):
            ref = dict(np.load(oracle_path))
            e32, e64 = errors_vs(g32, ref), errors_vs(g64, ref)
            out["vs_oracle"] = {"vs": "oracle_f64", "n": n_oracle, "steps": steps,
                                "oracle_seconds": float(ref["sec"]), "oracle_cores": _cores(),
                                "fp32": e32, "fp64": e64,
                                "fp32_h_bed_rel_l1_le_1e-5": bool(e32["h"]["rel_l1"] <= 1e-5 and
                                                                  e32["bed"]["rel_l1"] <= 1e-5)}
        else:
            out["vs_oracle"] = {"error": f"oracle process exit code {oracle_proc.exitcode}"}
    return out


def ensemble_run(count, steps, seed=0, world=1, rank=0):
    """The ragged ensemble: ``count`` dam breaks of random sizes advanced together, one
    launch per phase for all members, every member with its own dt.  With several ranks
    (replicas) the members are split over the ranks by ``partition_members`` and each rank
    advances its share; the whole-job rate is the sum of the ranks' cells over the slowest
    rank's time (two all-reduces of timing scalars, no data-path collective)."""
    import torch

    from pyexner_b200 import BoundaryManager, RoeExnerState
    from pyexner_b200.boundaries import index_coords
    from pyexner_b200.cases import ensemble_case, seds_matrix
    from pyexner_b200.ensemble import Ensemble, partition_members

    members, erosion = ensemble_case(count, seed)
    mine = partition_members([m["shape"][0] * m["shape"][1] for m in members], world)[rank]
    members = [members[k] for k in mine]
    seds = seds_matrix(erosion)
    mbs = []
    for m in members:
        ny, nx = m["shape"]
        X, Y = index_coords(ny, nx)
        mbs.append(dict(state=RoeExnerState.from_numpy(m["arrs"], seds, torch.float32),
                        boundaries=BoundaryManager(m["params"], X, Y), dx=m["dx"]))
    ens = Ensemble(mbs, erosion)
    ens.init()
    rows = ens.autotune()
    ens.run(3, "SSPRK2", 0.5)  # warm-up: captures the step graph
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    stream = torch.cuda.current_stream()
    e0.record(stream)
    dts = ens.run(steps, "SSPRK2", 0.5)
    e1.record(stream)
    e1.synchronize()
    sec = e0.elapsed_time(e1) / 1e3
    ens.check()
    cells = ens.cells()
    d = dts.double()
    cells_all, sec = sum_over_ranks(cells, world, "cuda"), max_over_ranks(sec, world, "cuda")
    return {"workload": f"roe_exner_ragged_ensemble_{count}_dambreaks_128-1024_mpm_ssprk2_f32",
            "members": count, "members_this_rank": len(mine), "cells": cells_all, "steps": steps,
            "value": cells_all * steps / sec, "unit": UNIT, "scaling": "strong" if world > 1 else None,
            "ms_per_step": 1e3 * sec / steps, "band_rows": rows, "launches_per_step": 4,
            "dt_range": [float(d.min()), float(d.max())], "l2": "state ~1.1 GB, larger than L2"}


def adjoint_run(n=512, steps=64, every=32):
    """Configuration 4's reverse mode (float64): ``steps`` SSPRK2 steps of the 512 x 512
    inflow case forward, then the checkpointed backward sweep with the parameter adjoints
    (discharge, sediment matrix); device time per step of each."""
    import torch

    from pyexner_b200 import BoundaryManager, RoeExnerState, cases, create_solver_bundle, run_steps
    from pyexner_b200.tangent import ParamAdjoints, vjp_init, vjp_run

    arrs, params, X, Y, target = cases.adjoint_case(n)
    bm = BoundaryManager(params, X, Y)
    raw = RoeExnerState.from_numpy(arrs, cases.seds_matrix(params["erosion"]), torch.float64)
    bundle = create_solver_bundle("Roe Exner")
    cfg = bundle.config(raw, None, bm, 0.01, params)
    mask = bundle.mask_fn(raw, None, bm.boundary_mask)
    st0 = bundle.init_fn(raw, mask, cfg)
    st = st0.clone()
    run_steps(st.clone(), mask, cfg, "SSPRK2", 2, 0.5, log_dt=False)  # graph capture
    torch.cuda.synchronize()
    e = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    e[0].record()
    run_steps(st, mask, cfg, "SSPRK2", steps, 0.5, log_dt=False)
    e[1].record()
    s = st.to_numpy()
    abar = raw.clone()
    for f in raw.PLANES:
        getattr(abar, f).zero_()
    g = np.zeros_like(s["z_b"])
    g[1:-1, 1:-1] = 2.0 * (s["z"] + s["z_b"] - target)[1:-1, 1:-1]
    abar.z_b.copy_(torch.from_numpy(g))
    pa = ParamAdjoints(cfg, raw.seds)
    torch.cuda.synchronize()
    e[2].record()
    vjp_run(st0, abar, mask, cfg, steps, "SSPRK2", 0.5, checkpoint_every=every, params=pa)
    vjp_init(raw, abar, mask, cfg, params=pa)
    e[3].record()
    e[3].synchronize()
    fwd, bwd = e[0].elapsed_time(e[1]) / steps, e[2].elapsed_time(e[3]) / steps
    return {"workload": f"roe_exner_inflow_{n}x{n}_mpm_ssprk2_f64_adjoint", "steps": steps,
            "checkpoint_every": every, "forward_ms_per_step": fwd, "backward_ms_per_step": bwd,
            "backward_over_forward": bwd / fwd,
            "note": "backward: checkpointed forward recomputation + reverse sweep with the discharge and "
                    "sediment-matrix adjoints, float64"}


def plain_roe_run(steps=200, cpu_steps=10):
    """The plain Roe dam-break, 256 x 256 cells, float64, SSPRK2, 200
    steps through ``run_steps`` (graph replay), and the float64 NumPy oracle on the host
    for ``cpu_steps`` steps of the same case (single thread)."""
    import torch

    from oracle import boundaries as OB
    from oracle import integrators as OI
    from pyexner_b200 import BoundaryManager, RoeState, cases, create_solver_bundle, run_steps

    c = cases.dambreak_roe(256)
    params = dict(flux_scheme="Roe", boundaries=c["params"]["boundaries"])
    bm = BoundaryManager(params, c["X"], c["Y"])
    st = RoeState.from_numpy(c["arrs"], torch.float64)
    bundle = create_solver_bundle("Roe")
    cfg = bundle.config(st, None, bm, c["dx"], params)
    mask = bundle.mask_fn(st)
    st = bundle.init_fn(st, mask, cfg)
    warm = st.clone()
    run_steps(warm, mask, cfg, "SSPRK2", steps, 0.5, log_dt=False)  # captures the step graph
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    run_steps(st, mask, cfg, "SSPRK2", steps, 0.5, log_dt=False)
    e1.record()
    e1.synchronize()
    sec = e0.elapsed_time(e1) / 1e3
    cells = 256 * 256
    obcs = OB.Boundaries("Roe", c["params"]["boundaries"], c["X"], c["Y"])
    arrs = {k: np.array(v) for k, v in c["arrs"].items()}
    t = time.perf_counter()
    OI.run_roe(arrs, obcs, c["dx"], 0.5, cpu_steps, "SSPRK2")
    cpu = cells * cpu_steps / (time.perf_counter() - t)
    return {"workload": "roe_dambreak_256x256_reflective_ssprk2_f64", "steps": steps, "value": cells * steps / sec,
            "unit": UNIT, "ms_per_step": 1e3 * sec / steps,
            "cpu_oracle": {"value": cpu, "unit": UNIT, "cores": 1, "kind": "port",
                           "sample": f"{cpu_steps} SSPRK2 steps of the same case, float64 NumPy oracle"}}


def _oracle_case(n, dtype=np.float64):
    from oracle import boundaries as OB
    from oracle import c_oracle as CO
    from pyexner_b200 import cases

    c = cases.gaussian_bed(n)
    bcs = OB.Boundaries("Roe Exner", c["params"]["boundaries"], c["X"], c["Y"])
    st = {k: np.array(v) for k, v in c["arrs"].items()}
    st["n_b"] = np.zeros_like(st["h"])
    st["seds"] = c["seds"]
    mask = OB.roe_exner_mask(st["z"].copy(), bcs.boundary_mask)
    st = CO.init(st, mask, bcs, True, c["dx"], dtype=dtype)
    return c, bcs, st, mask


def _cores():
    return int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))


def cpu_oracle_sample(n=2048, budget_s=10.0, min_steps=3, dtype=np.float32):
    """The C/OpenMP restatement of the reference step (all host threads) on the
    workload itself, SSPRK2 steps until ``budget_s`` seconds of CPU work."""
    from oracle import c_oracle as CO

    c, bcs, st, mask = _oracle_case(n, dtype)
    CO.run_roe_exner(st, mask, bcs, True, c["dx"], 0.5, 1, "SSPRK2", dtype=dtype)  # warm-up
    steps, sec = 0, 0.0
    while sec < budget_s or steps < min_steps:
        t0 = time.perf_counter()
        st, _ = CO.run_roe_exner(st, mask, bcs, True, c["dx"], 0.5, 1, "SSPRK2", dtype=dtype)
        sec += time.perf_counter() - t0
        steps += 1
    prec = "float32" if dtype == np.float32 else "float64"
    return n * n * steps / sec, _cores(), (f"{n}x{n} Gaussian-bed case (the workload), {steps} SSPRK2 steps, "
                                           f"{prec} C/OpenMP restatement of the reference step, {_cores()} threads")


def reference_arm(args):
    """The reference's algorithm on the host cores, on the workload itself (2048 x 2048):
    the C/OpenMP restatement of PyExner's step (JAX, which runs the reference itself, is
    not installed here) in float32, the precision the reference ships (its state is
    float32), with all host threads; one timed step = one SSPRK2 step.  The float64 build
    of the same restatement (the oracle) is timed beside it on a few steps."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import c_oracle as CO

    n = args.n
    c, bcs, st, mask = _oracle_case(n, np.float32)
    st, _ = CO.run_roe_exner(st, mask, bcs, True, c["dx"], 0.5, max(1, args.warmup), "SSPRK2", dtype=np.float32)
    t0 = time.perf_counter()
    st, _ = CO.run_roe_exner(st, mask, bcs, True, c["dx"], 0.5, args.steps, "SSPRK2", dtype=np.float32)
    sec = time.perf_counter() - t0
    v = n * n * args.steps / sec
    steps64 = max(2, args.steps // 5)
    c64, bcs64, st64, mask64 = _oracle_case(n, np.float64)
    CO.run_roe_exner(st64, mask64, bcs64, True, c64["dx"], 0.5, 1, "SSPRK2")
    t0 = time.perf_counter()
    CO.run_roe_exner(st64, mask64, bcs64, True, c64["dx"], 0.5, steps64, "SSPRK2")
    v64 = n * n * steps64 / (time.perf_counter() - t0)
    cores = _cores()
    sample = (f"{n}x{n} Gaussian-bed case (the workload itself), {args.warmup} + {args.steps} SSPRK2 steps, "
              f"float32 C/OpenMP restatement of the reference step, {cores} threads")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Gaussian bed)",
            "config": {"workload": f"roe_exner_gaussian_bed_{n}x{n}_mpm_ssprk2_f32", "cells": n * n},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "fp64_port": {"value": v64, "unit": UNIT, "steps": steps64, "cores": cores,
                          "sample": f"{n}x{n}, {steps64} SSPRK2 steps, float64 build (the oracle)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def oracle_reference_run(n, steps, path):
    """Float64 C/OpenMP oracle on the Gaussian-bed case at n x n for ``steps`` SSPRK2
    steps, final state to ``path`` (.npz).  Run in a spawned process beside the GPU work."""
    from oracle import c_oracle as CO

    c, bcs, st, mask = _oracle_case(n, np.float64)
    t0 = time.perf_counter()
    out, _ = CO.run_roe_exner(st, mask, bcs, True, c["dx"], 0.5, steps, "SSPRK2")
    np.savez(path, sec=time.perf_counter() - t0, **{k: out[k] for k in ("h", "hu", "hv", "z", "z_b")})


def errors_vs(a, ref):
    """rel-L1 and Linf (relative to max |ref|) of h, hu, hv and the total bed z + z_b over
    the physical cells."""
    s = (slice(1, -1), slice(1, -1))
    out = {}
    for name, x, y in (("h", a["h"], ref["h"]), ("hu", a["hu"], ref["hu"]), ("hv", a["hv"], ref["hv"]),
                       ("bed", a["z"] + a["z_b"], ref["z"] + ref["z_b"])):
        x, y = np.asarray(x, np.float64)[s], np.asarray(y, np.float64)[s]
        out[name] = {"rel_l1": float(np.sum(np.abs(x - y)) / max(np.sum(np.abs(y)), 1e-300)),
                     "linf": float(np.max(np.abs(x - y)) / max(np.max(np.abs(y)), 1e-300))}
    return out


def profile_sequence(args):
    import torch

    from pyexner_b200 import build, run_steps
    from pyexner_b200.integrators import check_state

    build.build()
    if args.profile_case == "roe":  # the plain Roe dam-break (256^2, float64)
        from pyexner_b200 import BoundaryManager, RoeState, cases, create_solver_bundle

        c = cases.dambreak_roe(256)
        params = dict(flux_scheme="Roe", boundaries=c["params"]["boundaries"])
        bm = BoundaryManager(params, c["X"], c["Y"])
        st = RoeState.from_numpy(c["arrs"], torch.float64)
        bundle = create_solver_bundle("Roe")
        cfg = bundle.config(st, None, bm, c["dx"], params)
        mask = bundle.mask_fn(st)
        st = bundle.init_fn(st, mask, cfg)
        run_steps(st, mask, cfg, "SSPRK2", max(1, args.warmup), 0.5, log_dt=False)
        torch.cuda.synchronize()
        if not bool(torch.isfinite(st.h).all()):
            raise SystemExit("plain Roe profile case: non-finite depth")
        return
    dt = torch.float32 if args.dtype == "f32" else torch.float64
    c, bundle, cfg, mask, st = build_case(args.n, dt, "cuda")
    run_steps(st, mask, cfg, "SSPRK2", max(1, args.warmup), 0.5)
    torch.cuda.synchronize()
    check_state(st, mask, cfg)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--impl", default="b200")
    ap.add_argument("--accuracy-steps", type=int, default=2000)
    ap.add_argument("--oracle-n", type=int, default=1024,
                    help="side of the accuracy case run by the float64 C oracle as well (0 to skip)")
    ap.add_argument("--n-big", type=int, default=8192, help="side of the bandwidth case (0 to skip)")
    ap.add_argument("--big-steps", type=int, default=20)
    ap.add_argument("--transport-u", type=float, default=1.0,
                    help="initial velocity of the bedload-everywhere variant of the case (0 to skip)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--adjoint-steps", type=int, default=64,
                    help="steps of the configuration-4 reverse-mode timing (0 to skip)")
    ap.add_argument("--ensemble-members", type=int, default=64, help="ragged ensemble size (0 to skip)")
    ap.add_argument("--ensemble-steps", type=int, default=1000)
    ap.add_argument("--profile", action="store_true",
                    help="short fixed sequence for ncu: build the case, run --warmup SSPRK2 steps, exit")
    ap.add_argument("--dtype", default="f32", choices=["f32", "f64"])
    ap.add_argument("--profile-case", default="gaussian", choices=["gaussian", "roe"],
                    help="case of --profile: the Gaussian-bed Roe-Exner grid or the plain Roe dam-break")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    if args.profile:
        return profile_sequence(args)

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    from pyexner_b200 import build

    if rank == 0:
        build.build()
    if world > 1:
        dist.barrier()

    n = args.n
    ncell = n * n
    flush = L2Flush()
    # ---- float32 device loop (replicas: every rank advances its own copy; no exchange)
    c, bundle, cfg, mask, st = build_case(n, torch.float32, "cuda")
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        sec, b = timed_device_loop(st, mask, cfg, args.steps, args.warmup, flush)
    sec = max_over_ranks(sec, world, "cuda")
    value = replica_throughput(world, ncell, args.steps, sec)
    kt = kernel_breakdown(st, b, mask, cfg, max(3, args.steps // 2), flush)
    hbm, peak_kind = peaks()
    esz = 4
    # per launch of re_stage_kernel, averaged over the two stages of a step
    stage_bytes = 0.5 * (WORDS_STAGE1 + WORDS_STAGE2) * esz * ncell
    stage_time = 0.5 * (kt["stage1"] + kt["stage2"])
    achieved = stage_bytes / stage_time / 1e9
    # DRAM bytes per launch of the stage kernel from the committed ncu summary (2048^2 case)
    traffic = None
    prof = os.path.join(ROOT, "profiles", "re_stage_f32_gaussian_bed_2048.md")
    if n == 2048 and os.path.exists(prof):
        tk = {}
        for line in open(prof):
            if line.startswith("traffic_bytes_stage"):
                k, val = line.split(":")
                tk[k.strip()] = float(val)
        if "traffic_bytes_stage1_2048" in tk and "traffic_bytes_stage2_2048" in tk:
            traffic = 0.5 * (tk["traffic_bytes_stage1_2048"] + tk["traffic_bytes_stage2_2048"])
    # ---- the 8192 x 8192 bandwidth case (same generator, 500-step configuration; K steps timed)
    big = None
    if args.n_big > 0:
        cb, bb, cfgb, maskb, stb = build_case(args.n_big, torch.float32, "cuda")
        secb, bscr = timed_device_loop(stb, maskb, cfgb, args.big_steps, args.warmup, flush)
        ktb = kernel_breakdown(stb, bscr, maskb, cfgb, max(3, args.big_steps // 2), flush)
        nb = args.n_big * args.n_big
        achb = 0.5 * (WORDS_STAGE1 + WORDS_STAGE2) * esz * nb / (0.5 * (ktb["stage1"] + ktb["stage2"])) / 1e9
        big = {"workload": f"roe_exner_gaussian_bed_{args.n_big}x{args.n_big}_mpm_ssprk2_f32",
               "value": nb * args.big_steps / secb, "unit": UNIT, "steps": args.big_steps,
               "roofline": {"achieved": achb, "peak": hbm, "unit": "GB/s", "frac": achb / hbm},
               "ms": {k: 1e3 * v for k, v in ktb.items()}}
        del stb, bscr
        torch.cuda.empty_cache()
    # ---- float64 device loop, same config
    c64, b64, cfg64, mask64, st64 = build_case(n, torch.float64, "cuda")
    sec64, _ = timed_device_loop(st64, mask64, cfg64, max(3, args.steps // 2), args.warmup, flush)
    value64 = ncell * max(3, args.steps // 2) / sec64
    del st64
    # ---- the same case with bedload everywhere (u0 = 1 m/s): the stage kernel's
    # sediment-free fast path never fires there
    transport = None
    if args.transport_u > 0:
        ct, bt, cfgt, maskt, stt = build_case(n, torch.float32, "cuda", u0=args.transport_u)
        sect, bscr = timed_device_loop(stt, maskt, cfgt, args.steps, args.warmup, flush)
        ktt = kernel_breakdown(stt, bscr, maskt, cfgt, max(3, args.steps // 2), flush)
        gpos = float((stt.G[1:-1, 1:-1] > 0).float().mean().item())
        transport = {"workload": f"roe_exner_gaussian_bed_{n}x{n}_mpm_ssprk2_f32_u{args.transport_u:g}",
                     "value": ncell * args.steps / sect, "unit": UNIT, "steps": args.steps,
                     "cells_with_bedload": gpos, "ms": {k: 1e3 * v for k, v in ktt.items()}}
        del stt, bscr
        torch.cuda.empty_cache()
    # ---- end to end through the public API with host buffers
    e2e_sec, h2d, d2h = e2e_run(n, torch.float32, args.steps, args.warmup)
    e2e_val = ncell * args.steps / e2e_sec
    # ---- CPU baseline (rank 0): the reference step's C restatement on the workload, while
    # the GPU is idle
    cpu = None
    if rank == 0 and not args.no_cpu:
        v, cores, sample = cpu_oracle_sample(n, 10.0)
        cpu = {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample}
    # ---- accuracy: the float64 oracle runs in a spawned process while the GPU works
    oracle_proc, oracle_path = None, None
    if rank == 0 and args.accuracy_steps > 0 and args.oracle_n > 0 and not args.no_cpu:
        import multiprocessing as mp
        import tempfile

        oracle_path = os.path.join(tempfile.mkdtemp(prefix="pxb_oracle_"), "ref.npz")
        oracle_proc = mp.get_context("spawn").Process(target=oracle_reference_run,
                                                      args=(args.oracle_n, args.accuracy_steps, oracle_path))
        oracle_proc.start()
    ens = (ensemble_run(args.ensemble_members, args.ensemble_steps, world=world, rank=rank)
           if args.ensemble_members > 0 else None)
    roe = plain_roe_run() if rank == 0 and not args.no_cpu else None
    adj = adjoint_run(steps=args.adjoint_steps) if rank == 0 and args.adjoint_steps > 0 else None
    acc = (accuracy_run(n, args.accuracy_steps, args.oracle_n, oracle_proc, oracle_path)
           if args.accuracy_steps > 0 else None)
    if rank != 0:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * sec / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Gaussian bed)",
        "config": {"workload": f"roe_exner_gaussian_bed_{n}x{n}_mpm_ssprk2_f32", "cells": ncell,
                   "parallelism": f"replicas{world}", "l2": "256 MiB write + 256 MiB read between timed steps (not timed)"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": traffic, "peak_kind": peak_kind,
                     "kernel": "re_stage_kernel, per launch (mean of the two SSPRK2 stages)",
                     "algorithmic_bytes_per_launch": stage_bytes,
                     "ms": {k: 1e3 * v for k, v in kt.items()}},
        "fp64": {"value": value64, "unit": UNIT, "fp32_over_fp64": value / world / value64},
        "bandwidth_case": big,
        "transport_case": transport,
        "ensemble": ens,
        "plain_roe": roe,
        "adjoint": adj,
        "accuracy": acc,
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d / args.steps,
                "d2h_bytes_per_step": d2h / args.steps,
                "note": "pinned host state -> device, init + K steps via run_steps, final state -> host "
                        "(second call; the first, untimed, warms the allocator and the step graph)"},
        "gpu_launches": 3 * args.steps,
        "clocks": clk.summary(),
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
