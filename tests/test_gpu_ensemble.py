"""Ragged ensembles (GPU only): every member of an ensemble run must give the bits of
the same member run on its own through ``run_steps`` — the per-item stage and CFL
bodies are shared, each member keeps its own dt, and the work decomposition (band
heights, which warp computes a cell) does not enter the arithmetic."""
import numpy as np
import pytest
import torch

from helpers import CASES, golden_re

pytestmark = pytest.mark.gpu

FIELDS = ("h", "hu", "hv", "z_b", "G")


@pytest.fixture(scope="module", autouse=True)
def _lib_built():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pyexner_b200 import build

    build.build()


def make_members(shapes, dtype, seed=3, extra=None):
    from pyexner_b200 import BoundaryManager, RoeExnerState, create_solver_bundle
    from pyexner_b200.boundaries import index_coords, ring_boundaries
    from pyexner_b200.cases import SED_ONE, ensemble_fields, seds_matrix

    erosion = dict(grass_factor="MPM", bulk_porosity=0.42, sediments=SED_ONE)
    rs = np.random.default_rng(seed)
    out = []
    for k, (nyp, nxp) in enumerate(shapes):
        arrs = ensemble_fields(nyp, nxp, float(rs.uniform(0.2, 1.0)), 0.01, seed_bed=seed * 100 + k)
        ny, nx = nyp + 2, nxp + 2
        # some momentum so that the first steps are not at rest
        arrs["hu"] = 0.2 * arrs["h"] * rs.uniform(-1, 1, arrs["h"].shape)
        bspec = ring_boundaries(ny, nx, ["Transmissive", "TransmissiveBed"], ["Transmissive", "TransmissiveBed"],
                                ["Reflective"], ["Reflective"])
        params = dict(flux_scheme="Roe Exner", erosion=erosion, boundaries=bspec)
        X, Y = index_coords(ny, nx)
        bm = BoundaryManager(params, X, Y)
        st = RoeExnerState.from_numpy(arrs, seds_matrix(erosion), dtype)
        out.append(dict(state=st, boundaries=bm, dx=0.01, params=params))
    if extra is not None:
        out.append(extra(dtype))
    return out, erosion


def single_runs(members, scheme, steps):
    """Each member on its own (fresh plan, init, run_steps)."""
    from pyexner_b200 import create_solver_bundle, run_steps

    res = []
    for mb in members:
        st = mb["state"].clone()
        bundle = create_solver_bundle("Roe Exner")
        cfg = bundle.config(st, None, mb["boundaries"], mb["dx"], mb["params"])
        mask = bundle.mask_fn(st, None, mb["boundaries"].boundary_mask)
        st = bundle.init_fn(st, mask, cfg)
        dts = run_steps(st, mask, cfg, scheme, steps, 0.5)
        res.append((st.to_numpy(), dts.cpu().numpy()))
    return res


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
@pytest.mark.parametrize("scheme,steps", [("SSPRK2", 4), ("FE", 5)])
def test_members_match_single_runs(dtype, scheme, steps):
    from pyexner_b200.ensemble import Ensemble

    members, erosion = make_members([(40, 60), (75, 33), (128, 97), (33, 150), (61, 61)], dtype)
    ref = single_runs(members, scheme, steps)
    ens = Ensemble(members, erosion, band_rows=16)
    ens.init()
    dts = ens.run(steps, scheme, 0.5).cpu().numpy()
    ens.check()
    for k, mb in enumerate(members):
        got = mb["state"].to_numpy()
        st_ref, dts_ref = ref[k]
        assert np.array_equal(dts[:, k], dts_ref), k
        for f in FIELDS:
            assert np.array_equal(got[f], st_ref[f]), (k, f)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
def test_large_members_take_items_from_the_work_queue(dtype):
    """Members large enough, with 8-row bands, that the ensemble's work items outnumber the
    resident warps several times over: a warp's first item is its index, the rest come
    from the ensemble kernel's queue, and members change under a warp between items.  The
    members must still give the bits of their single runs (which use the default bands)."""
    from pyexner_b200.ensemble import Ensemble

    members, erosion = make_members([(700, 650), (512, 700), (640, 600)], dtype, seed=9)
    ref = single_runs(members, "SSPRK2", 3)
    ens = Ensemble(members, erosion, band_rows=8)
    ens.init()
    dts = ens.run(3, "SSPRK2", 0.5).cpu().numpy()
    ens.check()
    for k, mb in enumerate(members):
        got = mb["state"].to_numpy()
        st_ref, dts_ref = ref[k]
        assert np.array_equal(dts[:, k], dts_ref), k
        for f in FIELDS:
            assert np.array_equal(got[f], st_ref[f]), (k, f)


def test_autotune_keeps_the_states_and_the_results():
    from pyexner_b200.ensemble import Ensemble

    members, erosion = make_members([(90, 70), (50, 130), (140, 40)], torch.float32, seed=5)
    ref = single_runs(members, "SSPRK2", 3)
    ens = Ensemble(members, erosion)
    ens.init()
    before = [mb["state"].to_numpy() for mb in members]
    rows = ens.autotune()
    assert rows in (8, 12, 16, 24, 32, 48, 64, 96, 128, 192, 256)
    for k, mb in enumerate(members):
        after = mb["state"].to_numpy()
        for f in FIELDS:
            assert np.array_equal(after[f], before[k][f])
    ens.run(3, "SSPRK2", 0.5)
    for k, mb in enumerate(members):
        got = mb["state"].to_numpy()
        for f in FIELDS:
            assert np.array_equal(got[f], ref[k][0][f]), (k, f)


def test_member_with_nodata_next_to_members_without(request):
    """A golden layout with nodata corners joins two plain members (mask planes are
    supplied for the members without one)."""
    from pyexner_b200 import BoundaryManager, RoeExnerState
    from pyexner_b200.ensemble import Ensemble

    case = [c for c in CASES if c[0] == "const_wetdry_nodata"][0]
    d, arrs, params, X, Y, mpm = golden_re(request.config.rootpath, case)

    def extra(dtype):
        bm = BoundaryManager(params, X, Y)
        st = RoeExnerState.from_numpy(arrs, d["seds"], dtype)
        return dict(state=st, boundaries=bm, dx=float(d["dx"]), params=params)

    for dtype in (torch.float64,):
        # constant grass factor for every member: the golden case is constant-G
        members, _ = make_members([(30, 44), (52, 27)], dtype, seed=9, extra=extra)
        for mb in members[:2]:
            mb["params"] = dict(mb["params"], erosion=params["erosion"])
            mb["state"].G.fill_(float(params["erosion"]["grass_factor"]))
        ref = single_runs(members, "SSPRK2", 3)
        ens = Ensemble(members, params["erosion"])
        ens.init()
        ens.run(3, "SSPRK2", 0.5)
        for k, mb in enumerate(members):
            got = mb["state"].to_numpy()
            for f in FIELDS:
                assert np.array_equal(got[f], ref[k][0][f]), (k, f)


def test_nonfinite_member_is_reported():
    from pyexner_b200 import PxbError
    from pyexner_b200.ensemble import Ensemble

    members, erosion = make_members([(30, 30), (40, 20), (25, 35)], torch.float64, seed=11)
    ens = Ensemble(members, erosion, band_rows=8)
    ens.init()
    members[1]["state"].hu[5, 5] = float("nan")
    ens.run(1, "SSPRK2", 0.5)
    with pytest.raises(PxbError) as ei:
        ens.check()
    assert ei.value.code == 3 and "member 1" in str(ei.value)
    ens.check()  # cleared


def test_unsupported_member_layout_is_refused():
    from pyexner_b200 import BoundaryManager, PxbError
    from pyexner_b200.boundaries import index_coords
    from pyexner_b200.ensemble import Ensemble

    members, erosion = make_members([(30, 30), (24, 20)], torch.float64, seed=2)
    mb = members[1]
    ny, nx = mb["state"].shape
    p = dict(mb["params"])
    p["boundaries"] = dict(p["boundaries"], inner={"type": "Transmissive", "polygon": [[9.5, 9.5], [10.5, 9.5],
                                                                                        [10.5, 10.5], [9.5, 10.5]],
                                                    "values": [0, 0, 0, 0], "normal": [1.0, 0.0]})
    X, Y = index_coords(ny, nx)
    mb["boundaries"] = BoundaryManager(p, X, Y)
    with pytest.raises(PxbError) as ei:
        Ensemble(members, erosion)
    assert ei.value.code == 4 and "member 1" in str(ei.value)
