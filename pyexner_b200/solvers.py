"""Solver bundles behind PyExner's plugin registry, computing on the B200 kernels.

Mirrors src/PyExner/solvers/registry.py:10-38: ``SolverConfig``, ``SolverBundle``,
``register_solver_bundle(name)`` and ``create_solver_bundle(name)``, with the bundles
"Roe Exner" (src/PyExner/solvers/roe_exner_solver.py) and "Roe"
(src/PyExner/solvers/roe_solver.py).  Signatures follow the Roe-Exner bundle, which is
the one PyExner's Forward Euler integrator drives (forwardeuler.py:39-40, 59, 97, 112):

    mask_fn(state, mpi_handler, b_mask) -> mask (2, ny, nx) bool on the device
    init_fn(state, mask, config)        -> state
    step_fn(state, time, dt, mask, config) -> state
    compute_dt_fn(state, cfl, mask, config) -> 0-d device tensor

Every compute call goes through the C ABI; there is no host fallback.  ``time`` reaches
the time-dependent handlers (Berthon, NormalFlowDepth).  A plan runs the fused stage
kernel when its boundary layout allows it and the general kernel chain otherwise
(``stage_path`` "auto"); "fused" or "general" force one.
"""
from __future__ import annotations

import ctypes
from typing import Callable, NamedTuple

import numpy as np
import torch

from . import _lib
from .boundaries import roe_exner_mask
from .state import alloc_plane


class SolverConfig(NamedTuple):
    mpi_handler: object
    boundaries: object
    dx: float
    halo_exchange: Callable = None
    compute_G: object = None  # "MPM" or the constant grass factor
    compute_n: object = None
    plans: dict = None        # plan cache of the config (per dtype / mask)
    band_rows: int = 0        # rows per warp band of the stage kernel (0 = sized to the device)
    stage_path: int = 0       # _lib.PATH_AUTO / PATH_FUSED / PATH_GENERAL


class SolverBundle(NamedTuple):
    name: str
    config: Callable
    mask_fn: Callable
    init_fn: Callable
    step_fn: Callable
    compute_dt_fn: Callable


SOLVER_REGISTRY: dict = {}


def register_solver_bundle(name):
    def decorator(bundle):
        SOLVER_REGISTRY[name] = bundle()
        return bundle()

    return decorator


def create_solver_bundle(name):
    bundle = SOLVER_REGISTRY.get(name)
    if bundle is None:
        raise ValueError(f"Unknown solver scheme '{name}'. Available options: {list(SOLVER_REGISTRY.keys())}")
    return bundle


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _identity(x):
    return x


def _dtype_code(t):
    if t == torch.float32:
        return _lib.F32
    if t == torch.float64:
        return _lib.F64
    raise ValueError(f"unsupported dtype {t}")


# ============================================================== Roe Exner
class RePlan:
    """Owner of one ``pxb_re_plan`` (boundary recipes, CFL scratch, graphs).

    ``workspace=True``: the plan's device memory is a torch tensor this object holds
    (``pxb_re_plan_create_in``), so the library allocates none for it."""

    def __init__(self, state, mask, config, band_rows=0, stage_path=0, workspace=False):
        ny, nx = state.shape
        self.mpm = isinstance(config.compute_G, str)
        nod = None
        m0 = mask[0] if mask is not None else None
        if m0 is not None and bool(m0.any()):
            nod = alloc_plane(ny, nx, torch.uint8, state.h.device, align=state.pitch)
            nod.copy_(m0.to(torch.uint8))
            if nod.stride(0) != state.pitch:
                raise ValueError("nodata plane pitch mismatch")
        self.nodata = nod
        self.seds = np.ascontiguousarray(np.asarray(state.seds, dtype=np.float64))
        handlers, nh = config.boundaries.c_array(state.pitch) if config.boundaries is not None else (None, 0)
        self._handlers = handlers
        cfg = _lib.REConfig()
        cfg.ny, cfg.nx, cfg.pitch = ny, nx, state.pitch
        cfg.dtype = _dtype_code(state.dtype)
        cfg.mpm = 1 if self.mpm else 0
        cfg.dx = float(config.dx)
        cfg.seds = self.seds.ctypes.data_as(ctypes.c_void_p) if self.mpm else None
        cfg.nsed = self.seds.shape[1] if self.mpm else 0
        cfg.nodata = nod.data_ptr() if nod is not None else None
        cfg.handlers = handlers if nh else None
        cfg.nhandlers = nh
        cfg.band_rows = int(band_rows)
        cfg.stage_path = int(stage_path)
        h = ctypes.c_void_p()
        self.workspace = None
        if workspace:
            size = ctypes.c_size_t()
            _lib.call("pxb_re_plan_workspace_size", ctypes.byref(cfg), ctypes.byref(size))
            # blocks of torch's caching allocator start on 512-byte boundaries
            self.workspace = torch.empty(max(1, size.value), dtype=torch.uint8, device=state.h.device)
            _lib.call("pxb_re_plan_create_in", ctypes.byref(cfg), ctypes.c_void_p(self.workspace.data_ptr()),
                      ctypes.c_size_t(self.workspace.numel()), ctypes.byref(h))
        else:
            _lib.call("pxb_re_plan_create", ctypes.byref(cfg), ctypes.byref(h))
        self.handle = h
        self.path = _lib.load().pxb_re_plan_path(h)
        self.dtype = state.dtype
        self.device = state.h.device

    def __del__(self):
        try:
            if getattr(self, "handle", None) is not None and self.handle.value:
                _lib.load().pxb_re_plan_destroy(self.handle)
        except Exception:
            pass

    def check(self):
        _lib.call("pxb_re_check", self.handle, _stream())


def _re_plan(state, mask, config):
    key = (state.dtype, state.shape, state.pitch, None if mask is None else mask.data_ptr())
    plans = config.plans
    if plans is None:
        return RePlan(state, mask, config, config.band_rows, config.stage_path)
    if key not in plans:
        plans[key] = RePlan(state, mask, config, config.band_rows, config.stage_path)
    return plans[key]


_PATHS = {"auto": _lib.PATH_AUTO, "fused": _lib.PATH_FUSED, "general": _lib.PATH_GENERAL}


def stage_path_code(v):
    """``stage_path`` parameter ("auto" / "fused" / "general" or the integer code)."""
    if isinstance(v, str):
        if v.lower() not in _PATHS:
            raise ValueError(f"unknown stage_path '{v}'. Available options: {list(_PATHS)}")
        return _PATHS[v.lower()]
    return int(v)


def get_mask(state, mpi_handler=None, b_mask=None):
    """roe_exner_solver.py:21-39 on one rank."""
    z = state.z.detach().cpu().numpy()
    bm = np.zeros(z.shape, bool) if b_mask is None else np.asarray(b_mask, bool)
    return torch.from_numpy(roe_exner_mask(z, bm)).to(state.h.device)


def config_fn_roeexner(state, mpi_handler, boundaries, dx, params):
    grass = params.get("erosion", {}).get("grass_factor", 0.0)
    return SolverConfig(mpi_handler=mpi_handler, boundaries=boundaries, dx=float(dx), halo_exchange=_identity,
                        compute_G=grass, compute_n=grass, plans={}, band_rows=int(params.get("band_rows", 0)),
                        stage_path=stage_path_code(params.get("stage_path", "auto")))


def init_fn_roeexner(state, mask, config):
    """roe_exner_solver.py:58-78: n_b, G and the handlers at t = 0 (on a copy)."""
    state.check_layout()
    out = state.clone()
    plan = _re_plan(out, mask, config)
    _lib.call("pxb_re_init", plan.handle, ctypes.byref(out.c_fields()), _stream())
    return out


def _dt_tensor(dt, state):
    if isinstance(dt, torch.Tensor):
        return dt.to(device=state.h.device, dtype=state.dtype).reshape(())
    return torch.tensor(float(dt), dtype=state.dtype, device=state.h.device)


def step_fn_roeexner(state, time, dt, mask, config, avg=None):
    """roe_exner_solver.py:80-116: one stage; with ``avg`` the SSPRK2 combination
    0.5*avg + 0.5*stage(state) is returned instead."""
    plan = _re_plan(state, mask, config)
    ny, nx = state.shape
    # the general path carries n through the handlers; the fused path leaves it as it is
    fields = ("h", "hu", "hv", "z_b", "G") + (("n",) if plan.path == _lib.PATH_GENERAL else ())
    new = {f: alloc_plane(ny, nx, state.dtype, state.h.device) for f in fields}
    out = state.replace(**new)
    dtt = _dt_tensor(dt, state)
    _lib.call("pxb_re_stage", plan.handle, ctypes.byref(state.c_fields()), ctypes.byref(out.c_fields()),
              ctypes.byref(avg.c_fields()) if avg is not None else None, ctypes.c_void_p(dtt.data_ptr()),
              float(time), _stream())
    return out


def compute_dt_roeexner(state, cfl, mask, config):
    """roe_exner_solver.py:118-122 (one rank): max(cfl * min_faces dt, 1e-6)."""
    plan = _re_plan(state, mask, config)
    dt = torch.empty((), dtype=state.dtype, device=state.h.device)
    _lib.call("pxb_re_cfl", plan.handle, ctypes.byref(state.c_fields()), float(cfl), ctypes.c_void_p(dt.data_ptr()),
              _stream())
    return dt


@register_solver_bundle("Roe Exner")
def solver_roeexner():
    return SolverBundle(name="Roe Exner", config=config_fn_roeexner, mask_fn=get_mask, init_fn=init_fn_roeexner,
                        step_fn=step_fn_roeexner, compute_dt_fn=compute_dt_roeexner)


# ============================================================== Roe
class RoePlan:
    def __init__(self, state, config):
        ny, nx = state.shape
        handlers, nh = config.boundaries.c_array(state.pitch) if config.boundaries is not None else (None, 0)
        self._handlers = handlers
        cfg = _lib.RoeConfig()
        cfg.ny, cfg.nx, cfg.pitch = ny, nx, state.pitch
        cfg.dtype = _dtype_code(state.dtype)
        cfg.dx = float(config.dx)
        cfg.handlers = handlers if nh else None
        cfg.nhandlers = nh
        h = ctypes.c_void_p()
        _lib.call("pxb_roe_plan_create", ctypes.byref(cfg), ctypes.byref(h))
        self.handle = h

    def __del__(self):
        try:
            if getattr(self, "handle", None) is not None and self.handle.value:
                _lib.load().pxb_roe_plan_destroy(self.handle)
        except Exception:
            pass

    def check(self):
        _lib.call("pxb_roe_check", self.handle, _stream())


def _roe_plan(state, config):
    key = (state.dtype, state.shape, state.pitch)
    if config.plans is None:
        return RoePlan(state, config)
    if key not in config.plans:
        config.plans[key] = RoePlan(state, config)
    return config.plans[key]


def get_mask_roe(state, *args, **kwargs):
    """roe_solver.py:14-17: ones on the interior (it does not restrict the CFL minimum)."""
    ny, nx = state.shape
    m = torch.zeros((ny, nx), dtype=state.dtype, device=state.h.device)
    m[1:-1, 1:-1] = 1
    return m


def config_fn_roe(state, mpi_handler, boundaries, dx, params):
    return SolverConfig(mpi_handler=mpi_handler, boundaries=boundaries, dx=float(dx), halo_exchange=_identity,
                        plans={})


def init_fn_roe(state, mask, config):
    """roe_solver.py:30-38: halo exchange only (a no-op on one device)."""
    return state.clone()


def step_fn_roe(state, time, dt, mask, config, avg=None):
    """roe_solver.py:40-54: update, then the handlers."""
    plan = _roe_plan(state, config)
    out = state.clone()  # z and n keep their interior values; ring cells are rewritten
    dtt = _dt_tensor(dt, state)
    _lib.call("pxb_roe_stage", plan.handle, ctypes.byref(state.c_fields()), ctypes.byref(out.c_fields()),
              ctypes.byref(avg.c_fields()) if avg is not None else None, ctypes.c_void_p(dtt.data_ptr()), _stream())
    return out


def compute_dt_roe(state, cfl, mask, config):
    """roe_solver.py:56-60: cfl * min over all cells; no floor."""
    plan = _roe_plan(state, config)
    dt = torch.empty((), dtype=state.dtype, device=state.h.device)
    _lib.call("pxb_roe_cfl", plan.handle, ctypes.byref(state.c_fields()), float(cfl), ctypes.c_void_p(dt.data_ptr()),
              _stream())
    return dt


@register_solver_bundle("Roe")
def solver_roe():
    return SolverBundle(name="Roe", config=config_fn_roe, mask_fn=get_mask_roe, init_fn=init_fn_roe,
                        step_fn=step_fn_roe, compute_dt_fn=compute_dt_roe)
