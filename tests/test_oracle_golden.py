"""Pin the oracle: it must reproduce the golden vectors made by running PyExner's
own code (tests/golden/make_golden.py) bit for bit."""
import numpy as np
import pytest

from bc_specs import BC_SPECS, ROE_BC_SPECS, grid_coords
from make_golden import CASES, ROE_CASES, NSTEPS
from oracle import boundaries as B
from oracle import integrators as I
from oracle import roe as R
from oracle import roe_exner as RE

GOLD = "tests/golden/"


def same(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    assert a.shape == b.shape
    ok = (a == b) | (np.isnan(a) & np.isnan(b))
    assert ok.all(), f"{np.count_nonzero(~ok)} of {a.size} differ; max |d| = {np.nanmax(np.abs(a - b))}"


@pytest.fixture(scope="module")
def faces(request):
    return np.load(request.config.rootpath / GOLD / "re_faces.npz")


@pytest.mark.parametrize("tag,normal", [("x", RE.NORMAL_X), ("y", RE.NORMAL_Y)])
def test_face_kernels(faces, tag, normal):
    f = faces
    si = (f["hi"], f["hui"], f["hvi"], f["zbi"], f["zi"], f["ni"])
    sj = (f["hj"], f["huj"], f["hvj"], f["zbj"], f["zj"], f["nj"])
    P, M = RE.roe_face(si, sj, normal, 0.1)
    same(np.stack(P, -1), f[f"roe_upwP_{tag}"])
    same(np.stack(M, -1), f[f"roe_upwM_{tag}"])
    se_i = (f["hi"], f["hui"], f["hvi"], f["zbi"], f["zi"], f["gi"])
    se_j = (f["hj"], f["huj"], f["hvj"], f["zbj"], f["zj"], f["gj"])
    same(RE.exner_face(se_i, se_j, normal), f[f"exner_F_{tag}"])
    sd_i = (f["hi"], f["hui"], f["hvi"], f["zi"], f["gi"])
    sd_j = (f["hj"], f["huj"], f["hvj"], f["zj"], f["gj"])
    same(RE.dt_face(sd_i, sd_j, normal, 0.1), f[f"dt_face_{tag}"])


def test_cubic(faces):
    lmin, lmax = RE._lambda_cubic(faces["cub_u"], faces["cub_a"], faces["cub_c"])
    same(lmin, faces["cub_lmin"])
    same(lmax, faces["cub_lmax"])


def test_cell_kernels(request):
    c = np.load(request.config.rootpath / GOLD / "re_cells.npz")
    for key in ("one", "two"):
        same(RE.compute_G_mpm(c["h"], c["hu"], c["hv"], c[f"seds_{key}"], c["mask"][0]), c[f"G_{key}"])
        same(RE.compute_n(c["n"], c["zb"], c[f"seds_{key}"]), c[f"nb_{key}"])
    same(RE.compute_G_const(c["h"], c["Gconst_in"], c["mask"][0]), c["Gconst"])


def load_re_case(root, case):
    name, (ny, nx), _regime, bcname, erosion = case
    d = np.load(root / GOLD / f"re_{name}.npz")
    X, Y = grid_coords(ny, nx)
    bcs = B.Boundaries("Roe Exner", BC_SPECS[bcname](ny, nx), X, Y)
    mask = B.roe_exner_mask(d["in_z"].copy(), bcs.boundary_mask)
    st = {k: d[f"in_{k}"] for k in ("h", "hu", "hv", "z", "z_b", "n", "G")}
    st["n_b"] = np.zeros_like(st["h"])
    st["seds"] = d["seds"]
    return d, bcs, mask, st, isinstance(erosion["grass_factor"], str)


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_roe_exner_step(request, case):
    d, bcs, mask, st, mpm = load_re_case(request.config.rootpath, case)
    same(mask, d["mask"])
    st = RE.init(st, mask, bcs, mpm)
    for k in RE.STATE_FIELDS:
        same(st[k], d[f"init_{k}"])
    dt = RE.compute_dt(st, 0.5, 0.1, mask[0])
    same(dt, d["dt0"])
    h, hu, hv, hu_c, hv_c = RE.hydro_and_corrections(st, dt, 0.1, mask)
    same(h, d["hydro_h"]); same(hu, d["hydro_hu"]); same(hv, d["hydro_hv"])
    same(hu_c, d["corr_hu"]); same(hv_c, d["corr_hv"])
    s1 = RE.stage(st, dt, 0.1, mask, bcs, mpm)
    for k in RE.STATE_FIELDS:
        same(s1[k], d[f"stage1_{k}"])
    for scheme, tag in (("FE", "fe"), ("SSPRK2", "rk")):
        out, dts = I.run_roe_exner(st, mask, bcs, mpm, 0.1, 0.5, NSTEPS, scheme)
        same(dts, d[f"{tag}_dts"])
        for k in RE.STATE_FIELDS:
            same(out[k], d[f"{tag}_{k}"])


@pytest.mark.parametrize("case", ROE_CASES, ids=[c[0] for c in ROE_CASES])
def test_roe_step(request, case):
    name, (ny, nx), _regime, bcname = case
    d = np.load(request.config.rootpath / GOLD / f"roe_{name}.npz")
    X, Y = grid_coords(ny, nx)
    bcs = B.Boundaries("Roe", ROE_BC_SPECS[bcname](ny, nx), X, Y)
    st = {k: d[f"in_{k}"] for k in R.FIELDS}
    dx = float(d["dx"])
    dt = R.compute_dt(st, 0.5, dx)
    same(dt, d["dt0"])
    s1 = R.stage(st, dt, dx, bcs)
    for k in R.FIELDS:
        same(s1[k], d[f"stage1_{k}"])
    out, dts = I.run_roe(st, bcs, dx, 0.5, NSTEPS, "SSPRK2")
    same(dts, d["rk_dts"])
    for k in R.FIELDS:
        same(out[k], d[f"rk_{k}"])


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
def test_c_oracle_matches_golden(request, case):
    """The C/OpenMP restatement (CPU baseline) against the same golden vectors."""
    from oracle import c_oracle as CO

    d, bcs, mask, st, mpm = load_re_case(request.config.rootpath, case)
    if any(hd.kind not in CO.KINDS for hd in bcs.handlers):
        pytest.skip("the C restatement carries the four boundary types of the benchmark layouts only")
    st = CO.init(st, mask, bcs, mpm, 0.1)

    def close(a, ref, rel, floor):
        # NaN (nodata beds) in the same places, relative error elsewhere
        assert np.array_equal(np.isnan(a), np.isnan(ref))
        ok = ~np.isnan(ref)
        if ok.any():
            assert np.max(np.abs(a[ok] - ref[ok])) <= rel * max(floor, np.max(np.abs(ref[ok])))

    for k in RE.STATE_FIELDS:
        close(st[k], d[f"init_{k}"], 1e-14, 1.0)
    for scheme, tag in (("FE", "fe"), ("SSPRK2", "rk")):
        out, dts = CO.run_roe_exner(st, mask, bcs, mpm, 0.1, 0.5, NSTEPS, scheme)
        assert np.max(np.abs(dts - d[f"{tag}_dts"])) <= 1e-15
        for k in RE.STATE_FIELDS:
            close(out[k], d[f"{tag}_{k}"], 1e-13, 1e-300)


@pytest.mark.parametrize("case", CASES[:3], ids=[c[0] for c in CASES[:3]])
def test_c_oracle_float32_build_tracks_golden(request, case):
    """The float32 build of the C restatement (the reference's own precision, timed by
    bench.py's reference arm) stays within float32 rounding of the float64 golden run."""
    from oracle import c_oracle as CO

    d, bcs, mask, st, mpm = load_re_case(request.config.rootpath, case)
    if any(hd.kind not in CO.KINDS for hd in bcs.handlers):
        pytest.skip("the C restatement carries the four boundary types of the benchmark layouts only")
    st = CO.init(st, mask, bcs, mpm, 0.1, dtype=np.float32)
    assert st["h"].dtype == np.float32
    out, dts = CO.run_roe_exner(st, mask, bcs, mpm, 0.1, 0.5, NSTEPS, "SSPRK2", dtype=np.float32)
    assert np.max(np.abs(dts - d["rk_dts"])) <= 1e-4 * np.max(np.abs(d["rk_dts"]))
    for k in ("h", "hu", "hv", "z_b"):
        ref = d[f"rk_{k}"]
        ok = ~np.isnan(ref)
        assert np.max(np.abs(out[k][ok] - ref[ok])) <= 1e-4 * max(1e-3, np.max(np.abs(ref[ok]))), k
