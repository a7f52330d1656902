"""pyexner_b200: PyExner's explicit finite-volume step on NVIDIA B200 (sm_100a).

The public surface mirrors PyExner's (src/PyExner/__init__.py): ``run_driver`` and the
state / solver / integrator registries.  Compute goes through ``libpyexner_b200.so``
(include/pyexner_b200.h); build it with ``python -m pyexner_b200.build``.
"""
from ._lib import PxbError
from .boundaries import BoundaryManager
from .integrators import (
    INTEGRATOR_REGISTRY,
    IntegratorBundle,
    IntegratorConfig,
    create_integrator_bundle,
    new_budget,
    outflow,
    register_integrator_bundle,
    run_steps,
    volume,
)
from .solvers import SOLVER_REGISTRY, SolverBundle, SolverConfig, create_solver_bundle, register_solver_bundle
from .state import STATE_REGISTRY, RoeExnerState, RoeState, create_state, register_state

__all__ = [
    "run_driver",
    "new_budget",
    "outflow",
    "volume",
    "BoundaryManager",
    "RoeState",
    "RoeExnerState",
    "STATE_REGISTRY",
    "create_state",
    "register_state",
    "SOLVER_REGISTRY",
    "SolverBundle",
    "SolverConfig",
    "create_solver_bundle",
    "register_solver_bundle",
    "INTEGRATOR_REGISTRY",
    "IntegratorBundle",
    "IntegratorConfig",
    "create_integrator_bundle",
    "register_integrator_bundle",
    "run_steps",
    "PxbError",
]


def run_driver(config_path):
    from .driver import run_driver as _rd

    return _rd(config_path)
