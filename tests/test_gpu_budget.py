"""Water and sediment volume budget of the Roe-Exner step (GPU only).

The reference advances every cell by flux differences: the fluctuations of each face are
scattered to its two cells (roe_exner.py:597-606) and the Exner face fluxes enter z_b with
opposite signs on the two sides (roe_exner.py:708-715).  Over the physical cells the
interior faces therefore telescope, and volume(end) - volume(start) + boundary outflow
vanishes up to rounding.  ``volume`` sums sum(h) dx^2 and sum(z_b) dx^2 in compensated
float64; ``run_steps(..., budget=...)`` accumulates the outflow through the boundary faces
as the fused stage kernel evaluates them.

Closed box (reflective walls all round): the mirrored wall states give a zero mass flux
up to rounding, so the water volume is conserved to rounding.  The sediment is not: at a
mirrored wall the reference's upwind speed is exactly 0 and its upwinding then takes the
left cell's bedload flux (roe_exner.py:645-661), which is not 0 when the wall-side cell
moves toward or away from the wall; the budget closes against those wall fluxes instead.
The flows here are subcritical and wet everywhere, so no face takes the Harten-Hyman
entropy fix, whose lambda_3 guard (roe_exner.py:371) is not mass conserving.
Tolerances: relative to the volume, 1e-13 in float64 and 1e-6 in float32 over 1000 steps.
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib_built():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pyexner_b200 import build

    build.build()


def gaussian_case(n, dtype, walls, u0, grass):
    """The Gaussian-bed generator with the given side handlers and grass factor."""
    from pyexner_b200 import BoundaryManager, RoeExnerState, cases, create_solver_bundle
    from pyexner_b200.boundaries import index_coords, ring_boundaries

    ny = nx = n + 2
    arrs = cases.gaussian_bed_fields(n, u0=u0)
    arrs["hv"] = 0.05 * arrs["h"]  # a y-velocity too, so that every wall sees flow
    if grass == "MPM":
        erosion = dict(grass_factor="MPM", bulk_porosity=0.42, sediments=cases.SED_ONE)
    else:
        erosion = dict(grass_factor=float(grass))
        arrs["G"] = np.full_like(arrs["h"], float(grass))
    if walls == "closed":
        bspec = ring_boundaries(ny, nx, ["Reflective"], ["Reflective"], ["Reflective"], ["Reflective"])
    else:
        bspec = ring_boundaries(ny, nx, ["Transmissive", "TransmissiveBed"], ["Transmissive", "TransmissiveBed"],
                                ["Reflective"], ["Reflective"])
    X, Y = index_coords(ny, nx)
    params = dict(flux_scheme="Roe Exner", erosion=erosion, boundaries=bspec)
    st = RoeExnerState.from_numpy(arrs, cases.seds_matrix(erosion), dtype)
    bundle = create_solver_bundle("Roe Exner")
    bm = BoundaryManager(params, X, Y)
    cfg = bundle.config(st, None, bm, 0.01, params)
    mask = bundle.mask_fn(st, None, bm.boundary_mask)
    st = bundle.init_fn(st, mask, cfg)
    return st, mask, cfg


TOL = {torch.float64: 1e-13, torch.float32: 1e-6}


def test_volume_matches_host_sum():
    from pyexner_b200 import volume

    st, mask, cfg = gaussian_case(126, torch.float64, "open", 0.1, "MPM")
    got = volume(st, mask, cfg)
    a = st.to_numpy()
    ref = (float(np.sum(a["h"][1:-1, 1:-1])) * 1e-4, float(np.sum(a["z_b"][1:-1, 1:-1])) * 1e-4)
    assert abs(got[0] - ref[0]) <= 1e-14 * ref[0]
    assert abs(got[1] - ref[1]) <= 1e-14 * ref[1]


@pytest.mark.parametrize("scheme", ["SSPRK2", "FE"])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
def test_closed_box_conserves_water(dtype, scheme):
    """Reflective walls all round, constant grass factor (bedload everywhere)."""
    from pyexner_b200 import new_budget, outflow, run_steps, volume

    st, mask, cfg = gaussian_case(126, dtype, "closed", 0.1, 0.005)
    w0, z0 = volume(st, mask, cfg)
    bud = new_budget()
    run_steps(st, mask, cfg, scheme, 1000, 0.5, budget=bud, log_dt=False)
    w1, z1 = volume(st, mask, cfg)
    ow, oz = outflow(bud)
    tol = TOL[dtype]
    assert abs(w1 - w0) <= tol * w0, (w1 - w0) / w0
    assert abs(w1 - w0 + ow) <= tol * w0, (w1 - w0 + ow) / w0
    assert abs(z1 - z0 + oz) <= tol * z0, (z1 - z0 + oz) / z0
    assert z1 != z0  # the bed did move through the walls (see the module docstring)


@pytest.mark.parametrize("scheme", ["SSPRK2", "FE"])
@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
def test_open_box_budget_closes(dtype, scheme):
    """The benchmark's layout (transmissive x, reflective y) started at 1 m/s: bedload in
    every cell (MPM), water and sediment leaving through the open sides."""
    from pyexner_b200 import new_budget, outflow, run_steps, volume

    st, mask, cfg = gaussian_case(126, dtype, "open", 1.0, "MPM")
    w0, z0 = volume(st, mask, cfg)
    bud = new_budget()
    run_steps(st, mask, cfg, scheme, 1000, 0.5, budget=bud, log_dt=False)
    w1, z1 = volume(st, mask, cfg)
    ow, oz = outflow(bud)
    tol = TOL[dtype]
    assert abs(ow) > 1e3 * tol * w0 and abs(oz) > 0  # the flow really crosses the boundary
    assert abs(w1 - w0 + ow) <= tol * w0, (w1 - w0 + ow) / w0
    assert abs(z1 - z0 + oz) <= tol * z0, (z1 - z0 + oz) / z0


def test_budget_leaves_the_state_unchanged():
    """A run with the budget gives the state of the same run without it, bit for bit."""
    from pyexner_b200 import new_budget, run_steps

    for dtype in (torch.float64, torch.float32):
        a, mask, cfg = gaussian_case(126, dtype, "open", 1.0, "MPM")
        b = a.clone()
        run_steps(a, mask, cfg, "SSPRK2", 20, 0.5)
        run_steps(b, mask, cfg, "SSPRK2", 20, 0.5, budget=new_budget())
        x, y = a.to_numpy(), b.to_numpy()
        for f in ("h", "hu", "hv", "z_b", "G"):
            assert np.array_equal(x[f], y[f]), (dtype, f)


def test_budget_refused_on_general_path():
    from pyexner_b200 import _lib, new_budget, run_steps

    st, mask, cfg = gaussian_case(30, torch.float64, "open", 1.0, "MPM")
    cfg = cfg._replace(stage_path=_lib.PATH_GENERAL, plans={})
    with pytest.raises(_lib.PxbError):
        run_steps(st, mask, cfg, "SSPRK2", 2, 0.5, budget=new_budget())
