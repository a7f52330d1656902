"""A run of n SSPRK2 steps against n runs of one step (GPU only).

``run_steps(n)`` replays the captured graph of one step (CFL launch, stage 1, averaging
stage) n times back to back, the stage and CFL work queues and the running speed
maximum reset by their kernels' last blocks between launches; n runs of one step replay
it once per call, each with its own dt log.  The two must give the same dts and the
same state bit for bit on every layout, band height and regime: nothing the kernels
carry from one launch to the next may leak into the arithmetic.
"""
import numpy as np
import pytest
import torch

from helpers import random_re_case

pytestmark = pytest.mark.gpu

PLANES = ("h", "hu", "hv", "z_b", "G")


@pytest.fixture(scope="module", autouse=True)
def _lib_built():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pyexner_b200 import build

    build.build()


def device_case(arrs, params, X, Y, dtype, dx=0.1):
    from pyexner_b200 import BoundaryManager, RoeExnerState, create_solver_bundle
    from pyexner_b200.cases import seds_matrix

    seds = seds_matrix(params["erosion"])
    bm = BoundaryManager(params, X, Y)
    st = RoeExnerState.from_numpy(arrs, seds, dtype)
    bundle = create_solver_bundle("Roe Exner")
    cfg = bundle.config(st, None, bm, dx, params)
    mask = bundle.mask_fn(st, None, bm.boundary_mask)
    return bundle.init_fn(st, mask, cfg), mask, cfg


def run_vs_single(st, mask, cfg, nsteps):
    from pyexner_b200 import run_steps

    a = st.clone()
    da = run_steps(a, mask, cfg, "SSPRK2", nsteps, 0.5).cpu().numpy()
    b = st.clone()
    db = np.concatenate([run_steps(b, mask, cfg, "SSPRK2", 1, 0.5).cpu().numpy() for _ in range(nsteps)])
    assert np.array_equal(da, db), np.flatnonzero(da != db)
    x, y = a.to_numpy(), b.to_numpy()
    for f in PLANES:
        assert np.array_equal(x[f], y[f], equal_nan=True), f


@pytest.mark.parametrize("shape,band_rows,regime,bc,mpm", [
    ((70, 100), 8, "fast", "trans_x_refl_y", True),
    ((131, 61), 16, "wetdry", "refl_all", True),
    ((57, 83), 9, "fast", "influx_left", False),
    ((64, 55), 7, "wetdry", "partial_nodata", False),
    ((40, 29), 5, "fast", "refl_first", True),
    ((66, 58), 11, "fast", "refl_self", True),
    ((3, 3), 4, "smooth", "refl_all", True),
    ((200, 3), 4, "smooth", "trans_x_refl_y", True),
    ((3, 200), 4, "smooth", "trans_x_refl_y", True),
    ((5, 257), 4, "fast", "refl_all", True),
    ((41, 27), 2, "fast", "trans_x_refl_y", True),
    ((300, 530), 0, "fast", "trans_x_refl_y", True),
])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64], ids=["f32", "f64"])
def test_run_matches_single_steps(shape, band_rows, regime, bc, mpm, dtype):
    """Strips and bands of many sizes (items of one row included: bands of 2 rows whose
    boundary strips split into halves), wet/dry fronts, nodata cells, inflow, MPM and
    constant grass factors: 10 steps in one run against 10 runs of one step."""
    ny, nx = shape
    arrs, params, X, Y, mpm = random_re_case(ny, nx, seed=ny * 31 + nx, regime=regime, bcname=bc, mpm=mpm)
    params["band_rows"] = band_rows
    st, mask, cfg = device_case(arrs, params, X, Y, dtype)
    run_vs_single(st, mask, cfg, 10)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64], ids=["f32", "f64"])
@pytest.mark.parametrize("u0", [0.1, 0.55, 1.0])
def test_run_matches_single_steps_gaussian_bed(u0, dtype):
    """The Gaussian-bed workload, below, at and above the Shields threshold (no, part and
    all of the cells carrying bedload, so both face-speed forms of the CFL reduction and
    both Exner paths of the stage run)."""
    from pyexner_b200 import cases

    c = cases.gaussian_bed(254, u0=u0)
    st, mask, cfg = device_case(c["arrs"], c["params"], c["X"], c["Y"], dtype, c["dx"])
    run_vs_single(st, mask, cfg, 12)
