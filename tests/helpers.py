"""Shared helpers of the parity tests: build a case for the oracle and for the device."""
import numpy as np

from bc_specs import BC_SPECS, ROE_BC_SPECS, grid_coords
from make_golden import CASES, ROE_CASES

from oracle import boundaries as OB
from oracle import roe_exner as ORE

RE_PLANES = ("h", "hu", "hv", "z", "z_b", "n", "n_b", "G")
ROE_PLANES = ("h", "hu", "hv", "z", "n")


def rel_err(a, b):
    """Normwise relative error max|a-b| / max|b| (absolute when b is all zero) over the
    finite entries of b; NaN (nodata beds) must sit in the same places (else inf)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    if not np.array_equal(np.isnan(a), np.isnan(b)):
        return np.inf
    ok = ~np.isnan(b)
    a, b = a[ok], b[ok]
    scale = np.max(np.abs(b)) if b.size else 0.0
    d = np.max(np.abs(a - b)) if b.size else 0.0
    return d / scale if scale > 0 else d


def l1_rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = np.sum(np.abs(b))
    return np.sum(np.abs(a - b)) / s if s > 0 else np.sum(np.abs(a - b))


def golden_re(root, case):
    name, (ny, nx), _regime, bcname, erosion = case
    d = np.load(root / "tests" / "golden" / f"re_{name}.npz")
    spec = BC_SPECS[bcname](ny, nx)
    X, Y = grid_coords(ny, nx)
    mpm = isinstance(erosion["grass_factor"], str)
    arrs = {k: d[f"in_{k}"] for k in ("h", "hu", "hv", "z", "z_b", "n", "G")}
    params = dict(flux_scheme="Roe Exner", boundaries=spec, erosion=erosion)
    return d, arrs, params, X, Y, mpm


def random_re_case(ny, nx, seed, regime="fast", bcname="trans_x_refl_y", mpm=True):
    """A bigger seeded Roe-Exner case (several warp strips and bands)."""
    rng = np.random.default_rng(seed)
    h = rng.uniform(0.2, 0.5, (ny, nx))
    vel = {"smooth": 0.3, "fast": 3.0, "wetdry": 1.5}[regime]
    u = rng.uniform(-vel, vel, (ny, nx))
    v = rng.uniform(-vel, vel, (ny, nx))
    z = rng.uniform(-0.1, 0.1, (ny, nx))
    zb = rng.uniform(0.0, 0.1, (ny, nx))
    pick = rng.random((ny, nx))
    zb[pick < 0.08] = 0.0
    if regime == "wetdry":
        dd = rng.random((ny, nx))
        h[dd < 0.15] = 0.0
        h[(dd >= 0.15) & (dd < 0.22)] = 5e-5
        z[dd < 0.15] += 0.6
    n = rng.uniform(0.0, 0.03, (ny, nx))
    if bcname == "l_domain":
        z[:6, -6:] = np.nan  # the block outside the L (bc_specs.l_domain)
    if mpm:
        erosion = dict(grass_factor="MPM", bulk_porosity=0.42,
                       sediments={"s1": dict(fraction=1.0, diameter=1.61e-3, density=2630.0, deposition_flux=0.0,
                                             erosion_flux=0.0)})
        G = np.zeros((ny, nx))
    else:
        erosion = dict(grass_factor=0.005)
        G = 0.005 * np.ones((ny, nx))
    arrs = dict(h=h, hu=h * u, hv=h * v, z=z, z_b=zb, n=n, G=G)
    params = dict(flux_scheme="Roe Exner", boundaries=BC_SPECS[bcname](ny, nx), erosion=erosion)
    X, Y = grid_coords(ny, nx)
    return arrs, params, X, Y, mpm


def oracle_setup(arrs, params, X, Y, mpm, seds):
    bcs = OB.Boundaries("Roe Exner", params["boundaries"], X, Y)
    mask = OB.roe_exner_mask(np.array(arrs["z"], copy=True), bcs.boundary_mask)
    st = {k: np.array(arrs[k], dtype=np.float64) for k in ("h", "hu", "hv", "z", "z_b", "n", "G")}
    st["n_b"] = np.zeros_like(st["h"])
    st["seds"] = seds
    st = ORE.init(st, mask, bcs, mpm)
    return st, mask, bcs


__all__ = ["CASES", "ROE_CASES", "ROE_BC_SPECS", "RE_PLANES", "ROE_PLANES", "rel_err", "l1_rel", "golden_re",
           "random_re_case", "oracle_setup", "grid_coords"]
