"""``run_driver``: the YAML front end (src/PyExner/runtime/driver.py:17-62) on one GPU.

Reads the same keys: end_time, out_freq, cfl, flux_scheme ("Roe" | "Roe Exner"),
integrator ("Forward Euler" | "SSPRK2"), input_file, output_file, erosion, boundaries.
MPI keys (parNx, parNy) must describe one rank.  Two keys are added: ``precision``
("fp32" default, or "fp64") and ``n_steps`` (run that many steps on the device instead of
the time-driven loop with output windows).
"""
from __future__ import annotations

import os

import yaml

from .boundaries import BoundaryManager
from .integrators import create_integrator_bundle
from .io import NetCDFStateIO
from .solvers import create_solver_bundle
from .state import STATE_REGISTRY


def run_driver(config_path):
    if isinstance(config_path, dict):
        params = dict(config_path)
        base = os.getcwd()
    else:
        with open(config_path, "r") as f:
            params = yaml.safe_load(f)
        base = os.path.dirname(os.path.abspath(config_path))
    if int(params.get("parNx", 1)) * int(params.get("parNy", 1)) != 1:
        raise ValueError("pyexner_b200 runs one domain per GPU: parNx * parNy must be 1")
    end_time = params.get("end_time", 1)
    out_freq = params.get("out_freq", 1)
    cfl = params.get("cfl", 0.5)
    flux_scheme = params.get("flux_scheme", "Roe")
    time_scheme = params.get("integrator", "Forward Euler")
    dtype = {"fp32": "float32", "fp64": "float64"}[params.get("precision", "fp32")]

    def path(p):
        return p if p is None or os.path.isabs(p) else os.path.join(base, p)

    io = NetCDFStateIO(path(params["input_file"]), path(params.get("output_file")))
    mesh = io.generate_mesh()
    state = io.read_state(STATE_REGISTRY[flux_scheme], mesh, params, dtype=dtype) if flux_scheme == "Roe Exner" else \
        STATE_REGISTRY[flux_scheme].from_numpy(_roe_arrays(io, mesh, params), dtype=dtype)
    boundaries = BoundaryManager(params, mesh.local_X, mesh.local_Y)
    solver = create_solver_bundle(flux_scheme)
    solver_config = solver.config(state, None, boundaries, mesh.dh, params)
    integrator = create_integrator_bundle(time_scheme)
    integrator_config = integrator.config(cfl, end_time, out_freq, solver, solver_config, params.get("n_steps"))
    state = integrator.run_fn(state, integrator_config, io, mesh, boundaries.boundary_mask)
    io.close()
    return state, (mesh.local_X, mesh.local_Y)


def _roe_arrays(io, mesh, params):
    from .state import RoeExnerState

    st = io.read_state(RoeExnerState, mesh, params, dtype="float64")
    return {k: getattr(st, k).cpu().numpy() for k in ("h", "hu", "hv", "z", "n")}
