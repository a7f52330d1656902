"""Integrator bundles behind PyExner's registry (src/PyExner/integrators/registry.py).

"Forward Euler" follows src/PyExner/integrators/forwardeuler.py:32-132 and "SSPRK2" the
intended form of src/PyExner/integrators/SSPRK2.py:30-51 (dt from u^n, two stages at the
same time argument, 0.5*u^n + 0.5*u^(2) on every leaf).

Two ways to run:
  * ``run_steps`` - a fixed number of steps, entirely on the device: the step (CFL
    reduction + stages) is captured once into a CUDA graph and replayed; dt never
    leaves the GPU (``pxb_re_run`` / ``pxb_roe_run``).  This is the timed hot path.
  * ``run_fn``    - the reference's time-driven loop with output windows.  Deciding
    when a window ends needs dt on the host, so this path synchronises once per step;
    it serves the YAML driver, not the benchmark.
"""
from __future__ import annotations

import ctypes
from typing import Callable, NamedTuple

import torch

from . import _lib
from .solvers import _re_plan, _roe_plan, _stream
from .state import RoeExnerState, alloc_plane

TIMESTEP_TOL = 5e-7  # src/utils/constants.py:25


class IntegratorConfig(NamedTuple):
    cfl: float
    end_time: float
    out_freq: float
    solver_config: object
    solver_bundle: object
    n_steps: int = None


class IntegratorBundle(NamedTuple):
    name: str
    config: Callable
    run_fn: Callable


INTEGRATOR_REGISTRY: dict = {}


def register_integrator_bundle(name):
    def decorator(bundle):
        INTEGRATOR_REGISTRY[name] = bundle()
        return bundle()

    return decorator


def create_integrator_bundle(name):
    bundle = INTEGRATOR_REGISTRY.get(name)
    if bundle is None:
        raise ValueError(f"Unknown integration scheme '{name}'. Available options: {list(INTEGRATOR_REGISTRY.keys())}")
    return bundle


def _config(cfl, end_time, out_freq, solver_bundle, solver_config, n_steps=None):
    return IntegratorConfig(cfl=cfl, end_time=end_time, out_freq=out_freq, solver_config=solver_config,
                            solver_bundle=solver_bundle, n_steps=n_steps)


def scratch_like(state):
    ny, nx = state.shape
    kw = {}
    for f in state.PLANES:
        kw[f] = alloc_plane(ny, nx, state.dtype, state.h.device)
    if isinstance(state, RoeExnerState):
        kw["seds"] = state.seds
    return type(state)(**kw)


def run_steps(state, mask, solver_config, scheme, n_steps, cfl, scratch=None, log_dt=True, t0=0.0, budget=None):
    """Advance ``state`` IN PLACE by ``n_steps`` steps on the device, starting at time
    ``t0`` (the step times are accumulated on the device).

    Returns the device tensor of the dts taken (or None).  ``scratch`` is a second
    state of the same layout (allocated when not given).  ``budget`` (Roe-Exner, fused
    stage path): a float64 device tensor from ``new_budget`` into which every step adds
    the water and sediment volume that left the physical cells through their boundary
    (read it with ``outflow``)."""
    code = _lib.SSPRK2 if scheme == "SSPRK2" else _lib.FE
    b = scratch if scratch is not None else scratch_like(state)
    dts = torch.empty(max(1, n_steps), dtype=state.dtype, device=state.h.device) if log_dt else None
    dptr = ctypes.c_void_p(dts.data_ptr()) if dts is not None else None
    if isinstance(state, RoeExnerState):
        plan = _re_plan(state, mask, solver_config)
        if budget is not None:
            if budget.dtype != torch.float64 or budget.numel() != 4 or budget.device != state.h.device:
                raise ValueError("budget must be the float64 device tensor of new_budget()")
            _lib.call("pxb_re_set_budget", plan.handle, ctypes.c_void_p(budget.data_ptr()))
        try:
            _lib.call("pxb_re_run", plan.handle, ctypes.byref(state.c_fields()), ctypes.byref(b.c_fields()),
                      int(n_steps), code, float(cfl), float(t0), dptr, _stream())
        finally:
            if budget is not None:
                _lib.call("pxb_re_set_budget", plan.handle, None)
    else:
        if budget is not None:
            raise ValueError("the volume budget is kept for Roe-Exner states")
        plan = _roe_plan(state, solver_config)
        _lib.call("pxb_roe_run", plan.handle, ctypes.byref(state.c_fields()), ctypes.byref(b.c_fields()),
                  int(n_steps), code, float(cfl), dptr, _stream())
    return dts[:n_steps] if dts is not None else None


def new_budget(device="cuda"):
    """A zeroed boundary-outflow accumulator for ``run_steps(..., budget=...)``: float64
    water and sediment outflow volumes (m^3), each with its compensation term."""
    return torch.zeros(4, dtype=torch.float64, device=device)


def outflow(budget):
    """(water, sediment) volumes (m^3) that left the physical cells, from ``budget``."""
    b = budget.detach().cpu().numpy()
    return float(b[0] + b[1]), float(b[2] + b[3])


def volume(state, mask, solver_config):
    """(water, erodible bed) volume in m^3 of the physical cells of a Roe-Exner state:
    sum h dx^2 and sum z_b dx^2 over rows and columns 1 .. n-2 that are not nodata,
    compensated float64 sums in a fixed order.  Together with the outflow of
    ``run_steps(..., budget=...)``, volume(end) - volume(start) + outflow is rounding."""
    plan = _re_plan(state, mask, solver_config)
    out = (ctypes.c_double * 2)()
    _lib.call("pxb_re_volume", plan.handle, ctypes.byref(state.c_fields()), out, _stream())
    return float(out[0]), float(out[1])


def autotune(state, mask, solver_config, scratch=None):
    """Time the fused stage kernel's band heights on ``state`` (left unchanged) and keep
    the fastest in the plan; returns it (0 on the general path)."""
    b = scratch if scratch is not None else scratch_like(state)
    plan = _re_plan(state, mask, solver_config)
    out = ctypes.c_int32(0)
    _lib.call("pxb_re_autotune", plan.handle, ctypes.byref(state.c_fields()), ctypes.byref(b.c_fields()), _stream(),
              ctypes.byref(out))
    return int(out.value)


def check_state(state, mask, solver_config):
    """Raise if a kernel flagged a non-finite dt or state value since the last check."""
    if isinstance(state, RoeExnerState):
        _re_plan(state, mask, solver_config).check()
    else:
        _roe_plan(state, solver_config).check()


def _ssprk2_step(bundle, st, t, dt, mask, cfg):
    s1 = bundle.step_fn(st, t, dt, mask, cfg)
    return bundle.step_fn(s1, t, dt, mask, cfg, avg=st)


def _run_time_loop(state, config, io, mesh, b_mask, ssprk2):
    """forwardeuler.py:51-132 on one device, with the time bookkeeping on the host.

    Inner window (the reference's device ``while_loop``, :32-49, :80): while
    ``time + dt_prev < target - TOL`` take a step with a fresh dt, where target is the
    next output time (capped at end_time) and dt_prev the last dt taken.  Then the
    window close (:85-117): a fresh dt; if it reaches the target a probe step of
    ``target - time`` is written out (not committed); the full step is always committed.
    SSPRK2 uses the same windows with two-stage steps.
    """
    bundle = config.solver_bundle
    cfg = config.solver_config
    mask = bundle.mask_fn(state, cfg.mpi_handler, b_mask)
    state = bundle.init_fn(state, mask, cfg)
    if config.n_steps is not None:
        run_steps(state, mask, cfg, "SSPRK2" if ssprk2 else "FE", config.n_steps, config.cfl)
        check_state(state, mask, cfg)
        return state

    def step(st, t, dt):
        return _ssprk2_step(bundle, st, t, dt, mask, cfg) if ssprk2 else bundle.step_fn(st, t, dt, mask, cfg)

    def target_of(t):
        return min((int(t / config.out_freq) + 1) * config.out_freq, config.end_time)

    if io is not None:
        io.write_state(state, mesh, mask[0])
    time, dt = 0.0, 0.0
    while time < config.end_time - TIMESTEP_TOL:
        while time + dt < target_of(time) - TIMESTEP_TOL:
            dt = float(bundle.compute_dt_fn(state, config.cfl, mask, cfg))
            state = step(state, time, dt)
            time += dt
        dt = float(bundle.compute_dt_fn(state, config.cfl, mask, cfg))
        target = target_of(time)
        if time + dt >= target - TIMESTEP_TOL:
            probe = step(state, time, target - time)
            if io is not None:
                io.write_state(probe, mesh, mask[0])
        state = step(state, time, dt)
        time += dt
    check_state(state, mask, cfg)
    return state


def run_fn_forwardeuler(state, config, io=None, mesh=None, b_mask=None):
    return _run_time_loop(state, config, io, mesh, b_mask, ssprk2=False)


def run_fn_ssprk2(state, config, io=None, mesh=None, b_mask=None):
    return _run_time_loop(state, config, io, mesh, b_mask, ssprk2=True)


@register_integrator_bundle("Forward Euler")
def integrator_forwardeuler():
    return IntegratorBundle(name="Forward Euler", config=_config, run_fn=run_fn_forwardeuler)


@register_integrator_bundle("SSPRK2")
def integrator_ssprk2():
    return IntegratorBundle(name="SSPRK2", config=_config, run_fn=run_fn_ssprk2)
