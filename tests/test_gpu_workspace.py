"""Roe-Exner plans inside a caller-owned workspace (GPU only).

``pxb_re_plan_workspace_size`` / ``pxb_re_plan_create_in``: the host framework owns the
plan's device memory (here a torch tensor), so that creating the plan and running its
init, CFL and stage calls allocate nothing in the library.  Checked: the same bits as a
plan on the library's own memory, no device memory taken beyond torch's (the driver's
free memory falls by exactly what torch reserves), the refusals of the entry points that
would allocate, and a workspace one byte short.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

PLANES = ("h", "hu", "hv", "z_b", "G")


@pytest.fixture(scope="module", autouse=True)
def _lib_built():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pyexner_b200 import build

    build.build()


def gaussian(n, dtype, stage_path):
    from pyexner_b200 import RoeExnerState, cases, create_solver_bundle

    c = cases.gaussian_bed(n, u0=1.0)
    params = dict(c["params"], stage_path=stage_path)
    st = RoeExnerState.from_numpy(c["arrs"], c["seds"], dtype)
    bundle = create_solver_bundle("Roe Exner")
    cfg = bundle.config(st, None, c["boundaries"], c["dx"], params)
    mask = bundle.mask_fn(st, None, c["boundaries"].boundary_mask)
    return bundle, st, mask, cfg


def with_plan(cfg, st, mask, workspace):
    """A config whose plan cache holds one plan for st (on a workspace or not)."""
    from pyexner_b200.solvers import RePlan

    plan = RePlan(st, mask, cfg, cfg.band_rows, cfg.stage_path, workspace=workspace)
    key = (st.dtype, st.shape, st.pitch, None if mask is None else mask.data_ptr())
    return cfg._replace(plans={key: plan}), plan


def steps(bundle, st, mask, cfg):
    """init, one dt, both SSPRK2 stages by the stage API, then 4 graph-replayed steps."""
    from pyexner_b200 import run_steps

    st = bundle.init_fn(st, mask, cfg)
    dt = bundle.compute_dt_fn(st, 0.5, mask, cfg)
    s1 = bundle.step_fn(st, 0.0, dt, mask, cfg)
    out = {"dt": np.float64(float(dt)), "s1": s1.to_numpy()}
    run_steps(st, mask, cfg, "SSPRK2", 4, 0.5)
    out["run"] = st.to_numpy()
    return out


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64], ids=["f32", "f64"])
@pytest.mark.parametrize("stage_path", ["fused", "general"])
def test_workspace_plan_gives_the_same_bits(dtype, stage_path):
    bundle, st, mask, cfg = gaussian(126, dtype, stage_path)
    cfg_a, plan_a = with_plan(cfg, st, mask, False)
    cfg_b, plan_b = with_plan(cfg, st, mask, True)
    assert plan_b.workspace is not None and plan_a.workspace is None
    a = steps(bundle, st.clone(), mask, cfg_a)
    b = steps(bundle, st.clone(), mask, cfg_b)
    assert a["dt"] == b["dt"]
    for k in ("s1", "run"):
        for f in PLANES:
            assert np.array_equal(a[k][f], b[k][f], equal_nan=True), (k, f)


def test_workspace_plan_allocates_nothing():
    """General path, float64, 1026^2: the seven scratch planes (59 MB) are the workspace's."""
    bundle, st, mask, cfg = gaussian(1024, torch.float64, "general")
    plane = st.h.stride(0) * st.h.shape[0] * 8
    # warm up every kernel the calls below launch (the driver sizes local memory on first use)
    cfg_w, _ = with_plan(cfg, st, mask, False)
    steps(bundle, st.clone(), mask, cfg_w)
    del cfg_w
    torch.cuda.synchronize()
    work = st.clone()
    torch.cuda.synchronize()

    def taken(make):
        free0, _ = torch.cuda.mem_get_info()
        res0 = torch.cuda.memory_reserved()
        obj = make()
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info()
        res1 = torch.cuda.memory_reserved()
        return obj, (free0 - free1) - (res1 - res0)  # device bytes taken outside torch

    def stage_calls(c):
        s = bundle.init_fn(work, mask, c)
        dt = bundle.compute_dt_fn(s, 0.5, mask, c)
        return bundle.step_fn(s, 0.0, dt, mask, c)

    (cfg_b, plan_b), extra = taken(lambda: with_plan(cfg, st, mask, True))
    assert extra == 0, extra
    _, extra = taken(lambda: stage_calls(cfg_b))
    assert extra == 0, extra
    (cfg_a, plan_a), extra = taken(lambda: with_plan(cfg, st, mask, False))
    assert extra >= 7 * plane, (extra, 7 * plane)


def test_workspace_plan_refusals():
    from pyexner_b200 import _lib, new_budget, run_steps
    from pyexner_b200.solvers import RePlan

    bundle, st, mask, cfg = gaussian(62, torch.float64, "fused")
    cfg_b, plan_b = with_plan(cfg, st, mask, True)
    st = bundle.init_fn(st, mask, cfg_b)
    with pytest.raises(_lib.PxbError):
        run_steps(st, mask, cfg_b, "SSPRK2", 2, 0.5, budget=new_budget())
    # one byte short of the size query
    c = _lib.REConfig()
    ny, nx = st.shape
    c.ny, c.nx, c.pitch, c.dtype, c.dx = ny, nx, st.pitch, _lib.F64, 0.01
    c.band_rows, c.stage_path = 0, _lib.PATH_FUSED
    size = ctypes.c_size_t()
    _lib.call("pxb_re_plan_workspace_size", ctypes.byref(c), ctypes.byref(size))
    assert size.value > 0
    ws = torch.empty(size.value, dtype=torch.uint8, device="cuda")
    h = ctypes.c_void_p()
    with pytest.raises(_lib.PxbError):
        _lib.call("pxb_re_plan_create_in", ctypes.byref(c), ctypes.c_void_p(ws.data_ptr()),
                  ctypes.c_size_t(size.value - 1), ctypes.byref(h))
    _lib.call("pxb_re_plan_create_in", ctypes.byref(c), ctypes.c_void_p(ws.data_ptr()), ctypes.c_size_t(size.value),
              ctypes.byref(h))
    assert _lib.load().pxb_re_plan_destroy(h) == 0
    assert isinstance(plan_b, RePlan)
