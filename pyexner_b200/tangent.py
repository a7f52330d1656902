"""Tangent-linear model of the float64 Roe-Exner step (forward-mode derivatives).

For a state ``u`` and a direction ``u_dot`` (a second RoeExnerState holding the tangent
of every plane), ``jvp_run`` advances both through ``n_steps`` integrator steps: the
values exactly as ``run_steps`` does in float64, the tangents by the chain rule through
every stage, including the dependence of dt on the state (through the fastest face).
This is what ``jax.jvp`` of the reference's loop would give.  The reverse mode
(``vjp_run`` / ``vjp_init``, further down) gives the gradient of a scalar objective with
respect to every plane of the initial state in one backward sweep.

``RoeExnerSteps`` wraps the run as a ``torch.autograd.Function`` with a forward-mode
rule, so ``torch.autograd.forward_ad`` dual tensors flow through it.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch
import torch.autograd.forward_ad as fwAD

from . import _lib
from .solvers import _re_plan, _stream
from .state import RoeExnerState, alloc_plane


def _check(state, state_dot):
    if state.dtype != torch.float64 or state_dot.dtype != torch.float64:
        raise ValueError("the tangent-linear model runs in float64")
    state.check_layout()
    state_dot.check_layout()
    if state_dot.pitch != state.pitch or state_dot.shape != state.shape:
        raise ValueError("state and tangent must share shape and pitch")


def _params(solver_config, seds_dot, inflow_dot):
    """``pxb_re_tangent_params`` for a tangent of the sediment matrix (7 x nsed, as the
    state's ``seds``) and of the discharges of ConstantInflux handlers (dict: boundary
    name -> tangent of its values[0])."""
    if seds_dot is None and not inflow_dot:
        return None, []
    keep = []
    p = _lib.TangentParams()
    if seds_dot is not None:
        sd = np.ascontiguousarray(np.asarray(seds_dot, dtype=np.float64))
        keep.append(sd)
        p.seds_dot = sd.ctypes.data
    if inflow_dot:
        names = [hd["name"] for hd in solver_config.boundaries.handlers]
        unknown = set(inflow_dot) - set(names)
        if unknown:
            raise KeyError(f"no boundary named {sorted(unknown)}")
        v = np.array([float(inflow_dot.get(n, 0.0)) for n in names], dtype=np.float64)
        keep.append(v)
        p.values0_dot = v.ctypes.data
    return p, keep


def jvp_init(state, state_dot, mask, solver_config, seds_dot=None, inflow_dot=None):
    """init_fn_roeexner and its tangent (on copies): returns (state, state_dot)."""
    _check(state, state_dot)
    s, t = state.clone(), state_dot.clone()
    plan = _re_plan(s, mask, solver_config)
    p, keep = _params(solver_config, seds_dot, inflow_dot)
    _lib.call("pxb_re_jvp_init", plan.handle, ctypes.byref(s.c_fields()), ctypes.byref(t.c_fields()),
              ctypes.byref(p) if p is not None else None, _stream())
    return s, t


def jvp_run(state, state_dot, mask, solver_config, n_steps, scheme="SSPRK2", cfl=0.5, t0=0.0, seds_dot=None,
            inflow_dot=None):
    """Advance ``state`` and ``state_dot`` IN PLACE by ``n_steps`` steps; returns the dts
    and their tangents as float64 device tensors.  ``seds_dot`` / ``inflow_dot``: tangents
    of the sediment matrix and of ConstantInflux discharges (see ``_params``)."""
    _check(state, state_dot)
    plan = _re_plan(state, mask, solver_config)
    p, keep = _params(solver_config, seds_dot, inflow_dot)
    dev = state.h.device
    dts = torch.empty(max(1, n_steps), dtype=torch.float64, device=dev)
    dts_dot = torch.empty(max(1, n_steps), dtype=torch.float64, device=dev)
    code = _lib.SSPRK2 if scheme == "SSPRK2" else _lib.FE
    _lib.call("pxb_re_jvp_run", plan.handle, ctypes.byref(state.c_fields()), ctypes.byref(state_dot.c_fields()),
              int(n_steps), code, float(cfl), float(t0), ctypes.byref(p) if p is not None else None,
              ctypes.c_void_p(dts.data_ptr()), ctypes.c_void_p(dts_dot.data_ptr()), _stream())
    return dts[:n_steps], dts_dot[:n_steps]


class StepsSpec:
    """What ``RoeExnerSteps`` runs: mask, solver config, sediment matrix, step count,
    scheme and CFL number."""

    def __init__(self, mask, solver_config, seds, n_steps, scheme="SSPRK2", cfl=0.5):
        self.mask, self.cfg, self.seds = mask, solver_config, seds
        self.n_steps, self.scheme, self.cfl = int(n_steps), scheme, float(cfl)


def _state_from(planes, seds):
    ny, nx = planes[0].shape
    kw = {}
    for f, p in zip(RoeExnerState.PLANES, planes):
        t = alloc_plane(ny, nx, torch.float64, planes[0].device)
        t.copy_(p)
        kw[f] = t
    return RoeExnerState(**kw, seds=seds)


class RoeExnerSteps(torch.autograd.Function):
    """``spec.n_steps`` fixed steps of the float64 Roe-Exner bundle as a differentiable
    function of the eight state planes (h, hu, hv, z, z_b, n, n_b, G).  Forward mode runs
    the tangent-linear kernels:

        with fwAD.dual_level():
            planes = [fwAD.make_dual(p, t) for p, t in zip(planes, tangents)]
            out = RoeExnerSteps.apply(spec, *planes)
            tangents_out = [fwAD.unpack_dual(o).tangent for o in out]

    and reverse mode (``loss.backward()``, ``torch.autograd.grad``) the adjoint kernels,
    which give gradients for h, hu, hv, z_b and G (z, n and n_b are held constant).
    """

    @staticmethod
    def forward(ctx, spec, *planes):
        from .integrators import run_steps

        ctx.spec = spec
        ctx.save_for_forward(*planes)
        ctx.save_for_backward(*planes)
        st = _state_from(planes, spec.seds)
        run_steps(st, spec.mask, spec.cfg, spec.scheme, spec.n_steps, spec.cfl, log_dt=False)
        return tuple(getattr(st, f).clone() for f in RoeExnerState.PLANES)

    @staticmethod
    def jvp(ctx, _spec_tangent, *tangents):
        spec = ctx.spec
        planes = ctx.saved_tensors
        st = _state_from(planes, spec.seds)
        td = _state_from([t if t is not None else torch.zeros_like(p) for t, p in zip(tangents, planes)], spec.seds)
        jvp_run(st, td, spec.mask, spec.cfg, spec.n_steps, spec.scheme, spec.cfl)
        return tuple(getattr(td, f).clone() for f in RoeExnerState.PLANES)

    @staticmethod
    def backward(ctx, *grads):
        spec = ctx.spec
        planes = ctx.saved_tensors
        st = _state_from(planes, spec.seds)
        abar = _state_from([g if g is not None else torch.zeros_like(p) for g, p in zip(grads, planes)], spec.seds)
        vjp_run(st, abar, spec.mask, spec.cfg, spec.n_steps, spec.scheme, spec.cfl)
        carried = ("h", "hu", "hv", "z_b", "G")
        return (None,) + tuple(getattr(abar, f).clone() if f in carried else None for f in RoeExnerState.PLANES)


__all__ = ["jvp_init", "jvp_run", "RoeExnerSteps", "StepsSpec", "fwAD"]


# ------------------------------------------------------------------ reverse mode
def _adj_fields(abar):
    return abar.c_fields()


class ParamAdjoints:
    """Adjoints of the scalar parameters, accumulated by ``vjp_run`` / ``vjp_init`` with
    ``params=``: ``seds_bar`` (7 x nsed like the state's ``seds``: dJ/d of the sediment
    matrix of pnetcdf_reader.py:136-158; row 1 is the grain diameter d50) and
    ``inflow_bar`` (boundary name -> dJ/d values[0], the discharge of each ConstantInflux
    handler).  The reverse-mode counterpart of ``jvp_run``'s ``seds_dot`` / ``inflow_dot``."""

    def __init__(self, solver_config, seds):
        handlers = solver_config.boundaries.handlers if solver_config.boundaries is not None else []
        self.names = [hd["name"] for hd in handlers]
        self.seds_bar = np.zeros(np.asarray(seds).shape, dtype=np.float64)
        self.values0_bar = np.zeros(max(1, len(self.names)), dtype=np.float64)

    @property
    def inflow_bar(self):
        return {n: float(v) for n, v in zip(self.names, self.values0_bar)}

    def _c(self):
        self.seds_bar = np.ascontiguousarray(self.seds_bar)
        p = _lib.ParamAdjoints()
        p.seds_bar = self.seds_bar.ctypes.data
        p.values0_bar = self.values0_bar.ctypes.data
        return p


def vjp_run(state0, abar, mask, solver_config, n_steps, scheme="SSPRK2", cfl=0.5, t0=0.0, checkpoint_every=32,
            params=None):
    """Reverse mode of ``n_steps`` fixed steps from ``state0`` (the state after init, not
    modified): ``abar`` (a RoeExnerState whose h, hu, hv, z_b, G hold dJ/du of the final
    state) is overwritten IN PLACE with dJ/du of ``state0``.  The run is redone forward
    with a checkpoint every ``checkpoint_every`` steps and undone segment by segment.
    ``params`` (a ParamAdjoints): also accumulate the parameter adjoints; then ``abar.n_b``
    (dJ/dn_b of the final state, n_b being constant) receives dJ/dn_b of ``state0``."""
    _check(state0, abar)
    plan = _re_plan(state0, mask, solver_config)
    code = _lib.SSPRK2 if scheme == "SSPRK2" else _lib.FE
    if params is None:
        _lib.call("pxb_re_vjp_run", plan.handle, ctypes.byref(state0.c_fields()), int(n_steps), code, float(cfl),
                  float(t0), int(checkpoint_every), ctypes.byref(_adj_fields(abar)), _stream())
    else:
        p = params._c()
        _lib.call("pxb_re_vjp_run_params", plan.handle, ctypes.byref(state0.c_fields()), int(n_steps), code,
                  float(cfl), float(t0), int(checkpoint_every), ctypes.byref(_adj_fields(abar)), ctypes.byref(p),
                  _stream())
    return abar


def vjp_init(state_raw, abar, mask, solver_config, params=None):
    """Reverse mode of init_fn_roeexner: ``abar`` (adjoint of the state after init) is
    overwritten IN PLACE with the adjoint of ``state_raw`` (the state before init).  With
    ``params``: also the parameter adjoints of the init, and ``abar.n_b`` (dJ/dn_b after
    init) goes through compute_n to ``abar.n`` and to the sediment matrix."""
    _check(state_raw, abar)
    plan = _re_plan(state_raw, mask, solver_config)
    if params is None:
        _lib.call("pxb_re_vjp_init", plan.handle, ctypes.byref(state_raw.c_fields()),
                  ctypes.byref(_adj_fields(abar)), _stream())
    else:
        p = params._c()
        _lib.call("pxb_re_vjp_init_params", plan.handle, ctypes.byref(state_raw.c_fields()),
                  ctypes.byref(_adj_fields(abar)), ctypes.byref(p), _stream())
    return abar


__all__ += ["vjp_run", "vjp_init", "ParamAdjoints"]
