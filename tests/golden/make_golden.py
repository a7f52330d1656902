"""Generate the golden vectors that pin the oracle to PyExner's own code.

Run (in the container that holds the reference checkout; not on the GPU box):

    python tests/golden/make_golden.py <checkout>/src/PyExner

It imports PyExner's modules from that source tree with ``jaxshim`` standing in for
``jax.numpy`` (float64 numpy, i.e. the reference's math with x64 enabled) and stubs
for ``mpi4py``/``mpi4jax``/``matplotlib`` (one rank: halo exchange and the dt
allreduce are identities).  It then runs the reference functions on small seeded
inputs and writes ``tests/golden/*.npz``.

What is executed is the reference's code, unmodified:
  * face kernels  ``roe_solver``, ``exner_solver``, ``compute_dt``, ``_get_lambda``
    (src/PyExner/solvers/kernels/roe_exner.py:163-255, 312-533, 614-663);
  * cell kernels  ``compute_G``, ``compute_n``, ``momentum_corrections``
    (roe_exner.py:14-130);
  * the "Roe Exner" bundle: ``get_mask``, ``config_fn_roeexner``,
    ``init_fn_roeexner``, ``step_fn_roeexner``, ``compute_dt_roeexner``
    (src/PyExner/solvers/roe_exner_solver.py:21-122);
  * the "Roe" kernels ``roe_solve_2D`` and ``compute_dt`` (src/PyExner/solvers/kernels/roe.py)
    and ``step_fn_roe`` / ``compute_dt_roe`` (src/PyExner/solvers/roe_solver.py:40-60);
  * ``BoundaryManager`` with the real handlers (src/PyExner/domain/boundary_registry.py).

Two integrator loops are restated here because the reference's cannot run as shipped:
  * Forward Euler as a fixed number of ``compute_dt_fn`` + ``step_fn`` pairs
    (src/PyExner/integrators/forwardeuler.py:37-49 without output probes);
  * SSPRK2 in its intended form (src/PyExner/integrators/SSPRK2.py:30-51):
    dt from u^n, two ``step_fn`` calls at the same time argument, then
    0.5*u^n + 0.5*u^(2) over every state leaf.  The shipped file imports names that
    do not exist and calls the bundle with the wrong arity.
"""
from __future__ import annotations

import dataclasses
import importlib
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import jaxshim  # noqa: E402

from bc_specs import BC_SPECS, ROE_BC_SPECS, grid_coords  # noqa: E402


def load_reference(src):
    jaxshim.install()
    pkg = types.ModuleType("PyExner")
    pkg.__path__ = [src]
    sys.modules["PyExner"] = pkg
    mods = types.SimpleNamespace()
    mods.k = importlib.import_module("PyExner.solvers.kernels.roe_exner")
    mods.kroe = importlib.import_module("PyExner.solvers.kernels.roe")
    mods.s = importlib.import_module("PyExner.solvers.roe_exner_solver")
    mods.sroe = importlib.import_module("PyExner.solvers.roe_solver")
    mods.b = importlib.import_module("PyExner.domain.boundary_registry")
    importlib.import_module("PyExner.domain.boundaries")
    mods.st = importlib.import_module("PyExner.state.roe_exner_state")
    mods.stroe = importlib.import_module("PyExner.state.roe_state")
    return mods


J = jaxshim.as_jarr


def mpi_one_rank():
    MPI = sys.modules["mpi4py.MPI"]
    return types.SimpleNamespace(
        coords=(0, 0),
        dims=(1, 1),
        rank=0,
        cart_comm=None,
        neighbors={d: MPI.PROC_NULL for d in ("north", "south", "east", "west")},
    )


# --------------------------------------------------------------------------- states
def make_state_arrays(rng, ny, nx, regime):
    """Seeded Roe-Exner input fields (with the ring) covering the branches of the step."""
    h = rng.uniform(0.2, 0.5, (ny, nx))
    vel = {"smooth": 0.3, "fast": 3.0, "wetdry": 1.5}[regime]
    u = rng.uniform(-vel, vel, (ny, nx))
    v = rng.uniform(-vel, vel, (ny, nx))
    z = rng.uniform(-0.1, 0.1, (ny, nx))
    zb = rng.uniform(0.0, 0.1, (ny, nx))
    n = rng.uniform(0.0, 0.03, (ny, nx))
    # sediment below SED_TOL in a few cells (exact zero and just below the threshold)
    pick = rng.random((ny, nx))
    zb[pick < 0.08] = 0.0
    zb[(pick >= 0.08) & (pick < 0.12)] = 5e-6
    if regime == "wetdry":
        d = rng.random((ny, nx))
        h[d < 0.15] = 0.0
        h[(d >= 0.15) & (d < 0.22)] = 5e-5  # below DRY_TOL but positive
        # a raised dry block: obstructs momentum in the corrections
        z[d < 0.15] += 0.6
    hu = h * u
    hv = h * v
    return dict(h=h, hu=hu, hv=hv, z=z, z_b=zb, n=n)


def l_block(arrs):
    """NaN bed in the top-right 6 x 6 block (the outside of an L-shaped domain)."""
    arrs["z"][:6, -6:] = np.nan
    return arrs


SEDS_MPM = {
    "one": {"s1": dict(fraction=1.0, diameter=1.61e-3, density=2630.0, deposition_flux=0.0, erosion_flux=0.0)},
    "two": {
        "s1": dict(fraction=0.6, diameter=1.0e-3, density=2650.0, deposition_flux=0.1, erosion_flux=0.2),
        "s2": dict(fraction=0.4, diameter=4.0e-3, density=2600.0, deposition_flux=0.3, erosion_flux=0.4),
    },
}


def seds_matrix(erosion):
    """The 7 x nsed matrix built by src/PyExner/io/pnetcdf_reader.py:136-162."""
    grass = erosion["grass_factor"]
    if isinstance(grass, str):
        rows = []
        for key in erosion["sediments"]:
            s = erosion["sediments"][key]
            rows.append([s["fraction"], s["diameter"], s["density"], s["deposition_flux"],
                         s["erosion_flux"], 0.047, erosion["bulk_porosity"]])
        return np.array(rows, dtype=np.float64).T
    return np.zeros((1, 1))


def initial_G(erosion, ny, nx):
    """src/PyExner/io/pnetcdf_reader.py:126-131."""
    grass = erosion["grass_factor"]
    if isinstance(grass, str):
        return np.zeros((ny, nx))
    return grass * np.ones((ny, nx))


CASES = [
    # name, (ny, nx), regime, bc spec, erosion, steps
    ("mpm1_smooth_tt", (11, 14), "smooth", "trans_x_refl_y", dict(grass_factor="MPM", bulk_porosity=0.42, sediments=SEDS_MPM["one"])),
    ("mpm1_fast_tt", (12, 13), "fast", "trans_x_refl_y", dict(grass_factor="MPM", bulk_porosity=0.42, sediments=SEDS_MPM["one"])),
    ("mpm2_wetdry_refl", (13, 11), "wetdry", "refl_all", dict(grass_factor="MPM", bulk_porosity=0.35, sediments=SEDS_MPM["two"])),
    ("const_fast_influx", (10, 15), "fast", "influx_left", dict(grass_factor=0.005)),
    ("const_wetdry_nodata", (12, 12), "wetdry", "partial_nodata", dict(grass_factor=0.01)),
    ("mpm1_fast_reflfirst", (11, 12), "fast", "refl_first", dict(grass_factor="MPM", bulk_porosity=0.42, sediments=SEDS_MPM["one"])),
    ("const_fast_selfrefl", (12, 14), "fast", "refl_self", dict(grass_factor=0.005)),
    ("const_smooth_berthon", (10, 16), "smooth", "berthon_like", dict(grass_factor=0.005)),
    ("mpm1_fast_outflux", (12, 15), "fast", "outflux_steep", dict(grass_factor="MPM", bulk_porosity=0.42, sediments=SEDS_MPM["one"])),
    ("mpm1_fast_ldomain", (14, 16), "fast", "l_domain", dict(grass_factor="MPM", bulk_porosity=0.42, sediments=SEDS_MPM["one"])),
]

DX = 0.1
CFL = 0.5
NSTEPS = 6


def state_from(mods, arrs, erosion):
    ny, nx = arrs["h"].shape
    return mods.st.RoeExnerState(
        h=J(arrs["h"]), hu=J(arrs["hu"]), hv=J(arrs["hv"]), z=J(arrs["z"]), z_b=J(arrs["z_b"]),
        n=J(arrs["n"]), n_b=J(np.zeros((ny, nx))), G=J(initial_G(erosion, ny, nx)),
        seds=J(seds_matrix(erosion)),
    )


FIELDS = ("h", "hu", "hv", "z", "z_b", "n", "n_b", "G")


def dump_state(prefix, st, out):
    for f in FIELDS:
        out[f"{prefix}_{f}"] = np.asarray(getattr(st, f), dtype=np.float64)


def ssprk2_average(a, b):
    kw = {}
    for fld in dataclasses.fields(a):
        kw[fld.name] = J(0.5 * np.asarray(getattr(a, fld.name)) + 0.5 * np.asarray(getattr(b, fld.name)))
    return type(a)(**kw)


def run_roe_exner_cases(mods):
    k, s = mods.k, mods.s
    for ci, (name, (ny, nx), regime, bcname, erosion) in enumerate(CASES):
        rng = np.random.default_rng(1000 + ci)
        arrs = make_state_arrays(rng, ny, nx, regime)
        if bcname == "l_domain":
            arrs = l_block(arrs)
        X, Y = grid_coords(ny, nx)
        params = dict(flux_scheme="Roe Exner", boundaries=BC_SPECS[bcname](ny, nx), erosion=erosion)
        bm = mods.b.BoundaryManager(params, J(X), J(Y))
        mpi = mpi_one_rank()
        st0 = state_from(mods, arrs, erosion)
        mask = s.get_mask(st0, mpi, bm.boundary_mask)
        cfg = s.config_fn_roeexner(st0, mpi, bm, DX, params)
        out = {"dx": np.float64(DX), "cfl": np.float64(CFL), "mask": np.asarray(mask)}
        for f in ("h", "hu", "hv", "z", "z_b", "n"):
            out[f"in_{f}"] = arrs[f]
        out["in_G"] = initial_G(erosion, ny, nx)
        out["seds"] = seds_matrix(erosion)
        st = s.init_fn_roeexner(st0, mask, cfg)
        dump_state("init", st, out)
        dt = s.compute_dt_roeexner(st, CFL, mask, cfg)
        out["dt0"] = np.float64(dt)
        # one stage (the unit the stage kernel replaces) and its sub-phases
        st_h = k.roe_solve_2D(st, dt, DX, mask)
        for f in ("h", "hu", "hv"):
            out[f"hydro_{f}"] = np.asarray(getattr(st_h, f))
        st_c = k.momentum_corrections(st_h, mask)
        for f in ("hu", "hv"):
            out[f"corr_{f}"] = np.asarray(getattr(st_c, f))
        st1 = s.step_fn_roeexner(st, 0.0, dt, mask, cfg)
        dump_state("stage1", st1, out)
        # Forward Euler, fixed step count; the time argument is the time at the step start
        fe = st
        dts = []
        t = 0.0
        for _ in range(NSTEPS):
            d = s.compute_dt_roeexner(fe, CFL, mask, cfg)
            fe = s.step_fn_roeexner(fe, t, d, mask, cfg)
            dts.append(float(d))
            t += float(d)
        out["fe_dts"] = np.array(dts)
        dump_state("fe", fe, out)
        # SSPRK2 (intended form): both stages at the time of the step start
        rk = st
        dts = []
        t = 0.0
        for _ in range(NSTEPS):
            d = s.compute_dt_roeexner(rk, CFL, mask, cfg)
            s1 = s.step_fn_roeexner(rk, t, d, mask, cfg)
            s2 = s.step_fn_roeexner(s1, t, d, mask, cfg)
            rk = ssprk2_average(rk, s2)
            dts.append(float(d))
            t += float(d)
        out["rk_dts"] = np.array(dts)
        dump_state("rk", rk, out)
        path = os.path.join(HERE, f"re_{name}.npz")
        np.savez_compressed(path, **out)
        print("wrote", path)


def run_face_kernels(mods):
    """Face-level outputs of the Roe-Exner kernels over seeded face pairs."""
    k = mods.k
    rng = np.random.default_rng(7)
    m = 400
    hi = rng.uniform(0.0, 0.6, m)
    hj = rng.uniform(0.0, 0.6, m)
    hi[:40] = 0.0
    hj[20:60] = 5e-5
    ui = rng.uniform(-4, 4, m)
    uj = rng.uniform(-4, 4, m)
    # transonic pairs for the Harten-Hyman fix: ei < 0 < ej
    uj[100:160] = np.sqrt(9.81 * np.maximum(hj[100:160], 1e-4)) * 1.5
    ui[100:160] = -np.sqrt(9.81 * np.maximum(hi[100:160], 1e-4)) * 0.5
    ui[160:220] = -np.sqrt(9.81 * np.maximum(hi[160:220], 1e-4)) * 1.5
    uj[160:220] = np.sqrt(9.81 * np.maximum(hj[160:220], 1e-4)) * 0.5
    vi = rng.uniform(-2, 2, m)
    vj = rng.uniform(-2, 2, m)
    zbi = rng.uniform(0, 0.1, m)
    zbj = rng.uniform(0, 0.1, m)
    zbi[::7] = 0.0
    zbj[3::11] = 4e-6
    zbj[250:270] = zbi[250:270] + 5e-6  # |dz_b| <= SED_TOL branch of the Exner speed
    zi = rng.uniform(-0.2, 0.2, m)
    zj = rng.uniform(-0.2, 0.2, m)
    ni = rng.uniform(0, 0.04, m)
    nj = rng.uniform(0, 0.04, m)
    gi = rng.uniform(0, 0.02, m)
    gj = rng.uniform(0, 0.02, m)
    gi[300:340] = 0.0
    gj[300:340] = 0.0
    out = {}
    arrays = dict(hi=hi, hj=hj, ui=ui, uj=uj, vi=vi, vj=vj, zbi=zbi, zbj=zbj, zi=zi, zj=zj,
                  ni=ni, nj=nj, gi=gi, gj=gj)
    out.update(arrays)
    hui, hvi, huj, hvj = hi * ui, hi * vi, hj * uj, hj * vj
    out.update(hui=hui, hvi=hvi, huj=huj, hvj=hvj)
    for tag, (nx_, ny_) in {"x": (1, 0), "y": (0, -1)}.items():
        si = (J(hi), J(hui), J(hvi), J(zbi), J(zi), J(ni))
        sj = (J(hj), J(huj), J(hvj), J(zbj), J(zj), J(nj))
        P, M = k.roe_solver(si, sj, nx_, ny_, DX)
        out[f"roe_upwP_{tag}"] = np.asarray(P)
        out[f"roe_upwM_{tag}"] = np.asarray(M)
        se_i = (J(hi), J(hui), J(hvi), J(zbi), J(zi), J(gi))
        se_j = (J(hj), J(huj), J(hvj), J(zbj), J(zj), J(gj))
        out[f"exner_F_{tag}"] = np.asarray(k.exner_solver(se_i, se_j, nx_, ny_, DX))
        sd_i = (J(hi), J(hui), J(hvi), J(zi), J(gi))
        sd_j = (J(hj), J(huj), J(hvj), J(zj), J(gj))
        out[f"dt_face_{tag}"] = np.asarray(k.compute_dt(sd_i, sd_j, nx_, ny_, DX))
    # the cubic on its own, over a sweep that includes the small-a fallback
    ut = rng.uniform(-3, 3, m)
    at = 10.0 ** rng.uniform(-8, 0.5, m)
    ct = rng.uniform(0.05, 3.0, m)
    lmin, lmax = k._get_lambda(J(ut), J(at), J(ct))
    out.update(cub_u=ut, cub_a=at, cub_c=ct, cub_lmin=np.asarray(lmin), cub_lmax=np.asarray(lmax))
    path = os.path.join(HERE, "re_faces.npz")
    np.savez_compressed(path, **out)
    print("wrote", path)


def run_cell_kernels(mods):
    k = mods.k
    rng = np.random.default_rng(11)
    ny, nx = 9, 10
    h = rng.uniform(0, 0.5, (ny, nx))
    h[::3, ::4] = 0.0
    hu = h * rng.uniform(-4, 4, (ny, nx))
    hv = h * rng.uniform(-4, 4, (ny, nx))
    zb = rng.uniform(0, 0.1, (ny, nx))
    zb[::5, 1::3] = 0.0
    n = rng.uniform(0, 0.03, (ny, nx))
    mask = np.zeros((2, ny, nx), bool)
    mask[0, 0, 0] = True
    mask[0, 4, 5] = True
    out = dict(h=h, hu=hu, hv=hv, zb=zb, n=n, mask=mask)
    for key, sed in SEDS_MPM.items():
        ero = dict(grass_factor="MPM", bulk_porosity=0.4, sediments=sed)
        seds = seds_matrix(ero)
        out[f"seds_{key}"] = seds
        out[f"G_{key}"] = np.asarray(k.compute_G(J(h), J(hu), J(hv), J(seds), mask))
        out[f"nb_{key}"] = np.asarray(k.compute_n(J(n), J(zb), J(seds)))
    gconst = k.compute_G_factory(True)
    g_in = rng.uniform(0, 0.02, (ny, nx))
    out["Gconst_in"] = g_in
    out["Gconst"] = np.asarray(gconst(J(h), J(hu), J(hv), None, mask, J(g_in)))
    path = os.path.join(HERE, "re_cells.npz")
    np.savez_compressed(path, **out)
    print("wrote", path)


ROE_CASES = [
    ("dambreak_refl", (18, 18), "dambreak", "roe_refl_all"),
    ("wet_trans", (12, 15), "wet", "roe_trans_x_refl_y"),
]


def run_roe_cases(mods):
    kroe, sroe = mods.kroe, mods.sroe
    for ci, (name, (ny, nx), regime, bcname) in enumerate(ROE_CASES):
        rng = np.random.default_rng(2000 + ci)
        if regime == "dambreak":
            xc = (np.arange(nx) + 0.5) / nx
            h = np.where(xc[None, :] < 0.5, 1.0, 0.1) * np.ones((ny, nx))
            hu = np.zeros((ny, nx))
            hv = np.zeros((ny, nx))
            z = np.zeros((ny, nx))
            n = np.zeros((ny, nx))
            dx = 1.0 / (nx - 2)
        else:
            h = rng.uniform(0.3, 1.0, (ny, nx))
            hu = h * rng.uniform(-0.5, 0.5, (ny, nx))
            hv = h * rng.uniform(-0.5, 0.5, (ny, nx))
            z = rng.uniform(-0.1, 0.1, (ny, nx))
            n = rng.uniform(0, 0.03, (ny, nx))
            dx = DX
        X, Y = grid_coords(ny, nx)
        params = dict(flux_scheme="Roe", boundaries=ROE_BC_SPECS[bcname](ny, nx))
        bm = mods.b.BoundaryManager(params, J(X), J(Y))
        mpi = mpi_one_rank()
        st0 = mods.stroe.RoeState(h=J(h), hu=J(hu), hv=J(hv), z=J(z), n=J(n))
        cfg = sroe.config_fn_roe(st0, mpi, bm, dx, params)
        mask = sroe.get_mask(st0)
        st = sroe.init_fn_roe(st0, cfg)
        out = {"dx": np.float64(dx), "cfl": np.float64(CFL)}
        for f in ("h", "hu", "hv", "z", "n"):
            out[f"in_{f}"] = np.asarray(getattr(st0, f))
        dt = sroe.compute_dt_roe(st, CFL, mask, cfg)
        out["dt0"] = np.float64(dt)
        st1 = sroe.step_fn_roe(st, 0.0, dt, cfg)
        for f in ("h", "hu", "hv", "z", "n"):
            out[f"stage1_{f}"] = np.asarray(getattr(st1, f))
        rk = st
        dts = []
        for _ in range(NSTEPS):
            d = sroe.compute_dt_roe(rk, CFL, mask, cfg)
            s1 = sroe.step_fn_roe(rk, 0.0, d, cfg)
            s2 = sroe.step_fn_roe(s1, 0.0, d, cfg)
            kw = {f: J(0.5 * np.asarray(getattr(rk, f)) + 0.5 * np.asarray(getattr(s2, f)))
                  for f in ("h", "hu", "hv", "z", "n")}
            rk = mods.stroe.RoeState(**kw)
            dts.append(float(d))
        out["rk_dts"] = np.array(dts)
        for f in ("h", "hu", "hv", "z", "n"):
            out[f"rk_{f}"] = np.asarray(getattr(rk, f))
        path = os.path.join(HERE, f"roe_{name}.npz")
        np.savez_compressed(path, **out)
        print("wrote", path)


def main():
    if len(sys.argv) < 2:
        raise SystemExit("usage: make_golden.py <path to the reference's src/PyExner>")
    src = sys.argv[1]
    mods = load_reference(src)
    np.seterr(all="ignore")
    run_face_kernels(mods)
    run_cell_kernels(mods)
    run_roe_exner_cases(mods)
    run_roe_cases(mods)


if __name__ == "__main__":
    main()
