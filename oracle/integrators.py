"""Fixed-step time integration loops for the oracle (test infrastructure only).

Forward Euler: src/PyExner/integrators/forwardeuler.py:37-49 (``body_fn``: dt from the
current state, then one ``step_fn``), run for a fixed step count without the
host-side output probes of forwardeuler.py:85-117.

SSPRK2: the intended form of src/PyExner/integrators/SSPRK2.py:30-51 (the shipped file
cannot run): dt from u^n, u1 = step(u^n, t, dt), u2 = step(u1, t, dt) with the same
time argument, u^{n+1} = 0.5*u^n + 0.5*u2 over every state leaf.
"""
from __future__ import annotations

import numpy as np

from . import roe as _roe
from . import roe_exner as _re


def _avg(a, b, fields):
    out = dict(a)
    for f in fields:
        out[f] = 0.5 * a[f] + 0.5 * b[f]
    return out


def run_roe_exner(st, mask, bcs, mpm, dx, cfl, nsteps, scheme, t0=0.0):
    """Fixed-step loop; the time argument of every stage is the time at the start of
    its step (SSPRK2.py:36-37 passes the same time to both stages)."""
    dts = []
    t = t0
    for _ in range(nsteps):
        dt = _re.compute_dt(st, cfl, dx, mask[0])
        if scheme == "SSPRK2":
            s1 = _re.stage(st, dt, dx, mask, bcs, mpm, t)
            s2 = _re.stage(s1, dt, dx, mask, bcs, mpm, t)
            st = _avg(st, s2, _re.STATE_FIELDS)
        else:
            st = _re.stage(st, dt, dx, mask, bcs, mpm, t)
        dts.append(float(dt))
        t = t + float(dt)
    return st, np.array(dts)


def run_roe(st, bcs, dx, cfl, nsteps, scheme):
    dts = []
    for _ in range(nsteps):
        dt = _roe.compute_dt(st, cfl, dx)
        if scheme == "SSPRK2":
            s1 = _roe.stage(st, dt, dx, bcs)
            s2 = _roe.stage(s1, dt, dx, bcs)
            st = _avg(st, s2, _roe.FIELDS)
        else:
            st = _roe.stage(st, dt, dx, bcs)
        dts.append(float(dt))
    return st, np.array(dts)
