"""Tangent-linear model (GPU only).

The dual run's values must be the float64 run's bits (same operations on the value
part), and its tangents must match central finite differences of the float64 device
run: on a smooth, fully wet case above the Shields threshold (no branch of the scheme
changes under the perturbation) the normwise relative difference must stay below 1e-6
for every plane after several steps (measured: about 5e-10 with eps = 1e-6), well inside
the 1e-4 the gradient checks ask for.  The dt tangent averages the faces that tie for the
maximum speed (mirror-image faces at reflective walls), as central differences do.
"""
import numpy as np
import pytest
import torch

from helpers import rel_err

pytestmark = pytest.mark.gpu

EVOLVING = ("h", "hu", "hv", "z_b", "G")


@pytest.fixture(scope="module", autouse=True)
def _lib_built():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pyexner_b200 import build

    build.build()


def smooth_case(ny=26, nx=34, layout="trans_x_refl_y"):
    """All wet, Froude ~0.6, Shields parameter well above its threshold everywhere, bed
    slopes far from the SED_TOL switch of the Exner speed."""
    from bc_specs import BC_SPECS, grid_coords

    r, c = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    h = 0.3 + 0.03 * np.sin(0.4 * c) * np.cos(0.3 * r)
    u = 1.0 + 0.1 * np.cos(0.25 * c + 0.2 * r)
    v = 0.15 * np.sin(0.3 * r)
    zb = 0.05 + 0.002 * c + 0.0015 * r
    erosion = dict(grass_factor="MPM", bulk_porosity=0.42,
                   sediments={"s1": dict(fraction=1.0, diameter=1.61e-3, density=2630.0, deposition_flux=0.0,
                                         erosion_flux=0.0)})
    arrs = dict(h=h, hu=h * u, hv=h * v, z=np.zeros_like(h), z_b=zb, n=np.full_like(h, 0.02), G=np.zeros_like(h))
    params = dict(flux_scheme="Roe Exner", boundaries=BC_SPECS[layout](ny, nx), erosion=erosion)
    X, Y = grid_coords(ny, nx)
    return arrs, params, X, Y


def setup(arrs, params, X, Y):
    from pyexner_b200 import BoundaryManager, RoeExnerState, create_solver_bundle
    from pyexner_b200.cases import seds_matrix

    bm = BoundaryManager(params, X, Y)
    st = RoeExnerState.from_numpy(arrs, seds_matrix(params["erosion"]), torch.float64)
    bundle = create_solver_bundle("Roe Exner")
    cfg = bundle.config(st, None, bm, 0.1, params)
    mask = bundle.mask_fn(st, None, bm.boundary_mask)
    st = bundle.init_fn(st, mask, cfg)
    return bundle, cfg, mask, st


def tangent_state(st, rng, planes=("h", "z_b")):
    t = st.clone()
    for f in st.PLANES:
        getattr(t, f).zero_()
    ny, nx = st.shape
    r, c = np.meshgrid(np.arange(ny), np.arange(nx), indexing="ij")
    for f in planes:
        scale = float(getattr(st, f).abs().max())
        field = scale * (np.sin(0.5 * c + rng.uniform(0, 3)) * np.cos(0.35 * r + rng.uniform(0, 3)))
        getattr(t, f).copy_(torch.from_numpy(field))
    return t


def perturbed(st, t, eps):
    s = st.clone()
    for f in st.PLANES:
        getattr(s, f).add_(eps * getattr(t, f))
    return s


@pytest.mark.parametrize("scheme", ["SSPRK2", "FE"])
def test_values_are_the_float64_run(scheme):
    from pyexner_b200 import run_steps
    from pyexner_b200.tangent import jvp_run

    bundle, cfg, mask, st = setup(*smooth_case())
    ref = st.clone()
    dts_ref = run_steps(ref, mask, cfg, scheme, 5, 0.5).cpu().numpy()
    t = tangent_state(st, np.random.default_rng(1))
    s = st.clone()
    dts, _ = jvp_run(s, t, mask, cfg, 5, scheme, 0.5)
    assert np.array_equal(dts.cpu().numpy(), dts_ref)
    a, b = s.to_numpy(), ref.to_numpy()
    for f in EVOLVING + ("n",):
        assert np.array_equal(a[f], b[f]), f


@pytest.mark.parametrize("scheme,planes", [("SSPRK2", ("h", "z_b")), ("SSPRK2", ("hu",)), ("FE", ("z_b",))])
def test_tangent_matches_central_differences(scheme, planes):
    from pyexner_b200 import run_steps
    from pyexner_b200.tangent import jvp_run

    bundle, cfg, mask, st = setup(*smooth_case())
    t = tangent_state(st, np.random.default_rng(7), planes)
    s, td = st.clone(), t.clone()
    dts, dts_dot = jvp_run(s, td, mask, cfg, 8, scheme, 0.5)
    eps = 1e-6
    runs = []
    for sign in (1.0, -1.0):
        p = perturbed(st, t, sign * eps)
        d = run_steps(p, mask, cfg, scheme, 8, 0.5)
        runs.append((p.to_numpy(), d.cpu().numpy()))
    got = td.to_numpy()
    for f in EVOLVING:
        fd = (runs[0][0][f] - runs[1][0][f]) / (2 * eps)
        assert rel_err(got[f], fd) <= 1e-6, (f, rel_err(got[f], fd))
    fd_dt = (runs[0][1] - runs[1][1]) / (2 * eps)
    assert np.max(np.abs(dts_dot.cpu().numpy() - fd_dt)) <= 1e-6 * max(1e-12, np.max(np.abs(fd_dt))) + 1e-14


def test_tangent_is_linear_in_the_direction():
    from pyexner_b200.tangent import jvp_run

    bundle, cfg, mask, st = setup(*smooth_case(layout="refl_all"))
    rng = np.random.default_rng(3)
    t1, t2 = tangent_state(st, rng), tangent_state(st, rng, ("hv", "z_b"))
    t12 = t1.clone()
    for f in st.PLANES:
        getattr(t12, f).mul_(2.0).add_(getattr(t2, f))
    outs = []
    for t in (t1, t2, t12):
        s, td = st.clone(), t.clone()
        jvp_run(s, td, mask, cfg, 4, "SSPRK2", 0.5)
        outs.append(td.to_numpy())
    for f in EVOLVING:
        assert rel_err(outs[2][f], 2 * outs[0][f] + outs[1][f]) <= 1e-11, f


def test_init_tangent_and_general_layout():
    """Through init (G from MPM) and the general path's time-dependent handlers."""
    from pyexner_b200 import BoundaryManager, RoeExnerState, create_solver_bundle, run_steps
    from pyexner_b200.cases import seds_matrix
    from pyexner_b200.tangent import jvp_init, jvp_run

    arrs, params, X, Y = smooth_case(24, 40, layout="berthon_like")
    params["erosion"] = dict(grass_factor=0.005)
    arrs["G"] = np.full_like(arrs["h"], 0.005)
    bm = BoundaryManager(params, X, Y)
    raw = RoeExnerState.from_numpy(arrs, seds_matrix(params["erosion"]), torch.float64)
    bundle = create_solver_bundle("Roe Exner")
    cfg = bundle.config(raw, None, bm, 0.1, params)
    mask = bundle.mask_fn(raw, None, bm.boundary_mask)
    t = tangent_state(raw, np.random.default_rng(5), ("h", "hu", "z_b"))
    s, td = jvp_init(raw, t, mask, cfg)
    ref = bundle.init_fn(raw, mask, cfg)
    for f in raw.PLANES:
        assert np.array_equal(s.to_numpy()[f], ref.to_numpy()[f]), f
    jvp_run(s, td, mask, cfg, 6, "SSPRK2", 0.5, t0=2.0)
    eps = 1e-6
    outs = []
    for sign in (1.0, -1.0):
        p = bundle.init_fn(perturbed(raw, t, sign * eps), mask, cfg)
        run_steps(p, mask, cfg, "SSPRK2", 6, 0.5, t0=2.0)
        outs.append(p.to_numpy())
    got = td.to_numpy()
    for f in ("h", "hu", "hv", "z_b"):
        fd = (outs[0][f] - outs[1][f]) / (2 * eps)
        assert rel_err(got[f], fd) <= 1e-6, (f, rel_err(got[f], fd))


def test_torch_forward_ad_through_the_function():
    import torch.autograd.forward_ad as fwAD

    from pyexner_b200.tangent import RoeExnerSteps, StepsSpec, jvp_run

    bundle, cfg, mask, st = setup(*smooth_case())
    t = tangent_state(st, np.random.default_rng(11))
    spec = StepsSpec(mask, cfg, st.seds, 3, "SSPRK2", 0.5)
    planes = [getattr(st, f).clone() for f in st.PLANES]
    tangents = [getattr(t, f).clone() for f in st.PLANES]
    with fwAD.dual_level():
        duals = [fwAD.make_dual(p, q) for p, q in zip(planes, tangents)]
        out = RoeExnerSteps.apply(spec, *duals)
        got = {f: fwAD.unpack_dual(o).tangent.cpu().numpy() for f, o in zip(st.PLANES, out)}
    s, td = st.clone(), t.clone()
    jvp_run(s, td, mask, cfg, 3, "SSPRK2", 0.5)
    ref = td.to_numpy()
    for f in EVOLVING:
        assert np.array_equal(got[f], ref[f]), f


def test_parameter_tangents_grain_size_and_inflow():
    """Tangents with respect to the grain diameter (sediment matrix row 1) and to the
    discharge of a ConstantInflux inlet, against central differences of runs whose plans
    are built from the perturbed parameters.  The discharge is a float32 value (as the
    reference parses boundary values), so its difference step is 1e-3 (the float32 rounding
    of a smaller step would dominate) and the tolerance the gradient checks' 1e-4.  A step
    that large moves the velocity field enough to cross faces where the Exner upwind
    direction switches (the sign of dq_b/dz_b changes where v changes sign), where the bed
    update jumps; so for the discharge the bed itself is not differenced: h, hu, hv and G
    are."""
    import copy

    from pyexner_b200 import BoundaryManager, RoeExnerState, create_solver_bundle, run_steps
    from pyexner_b200.cases import seds_matrix
    from pyexner_b200.tangent import jvp_init, jvp_run

    arrs, params, X, Y = smooth_case(layout="influx_left")

    def build(p):
        bm = BoundaryManager(p, X, Y)
        st = RoeExnerState.from_numpy(arrs, seds_matrix(p["erosion"]), torch.float64)
        bundle = create_solver_bundle("Roe Exner")
        cfg = bundle.config(st, None, bm, 0.1, p)
        mask = bundle.mask_fn(st, None, bm.boundary_mask)
        return bundle, cfg, mask, st

    def with_params(d_scale, q_shift):
        p = copy.deepcopy(params)
        p["erosion"]["sediments"]["s1"]["diameter"] *= d_scale
        p["boundaries"]["inlet"]["values"][0] += q_shift
        return p

    d0 = params["erosion"]["sediments"]["s1"]["diameter"]
    # d50 moves h only through the bed: its tangent there is small, so rounding noise of the
    # differences is relatively larger (1e-5)
    for which, eps, tol in (("d50", 1e-6, 1e-5), ("q", 1e-3, 1e-4)):
        bundle, cfg, mask, raw = build(params)
        zero = raw.clone()
        for f in raw.PLANES:
            getattr(zero, f).zero_()
        sd = np.zeros_like(raw.seds)
        kw = {}
        if which == "d50":
            sd[1, 0] = d0  # direction: d -> d (1 + eps)
            kw["seds_dot"] = sd
        else:
            kw["inflow_dot"] = {"inlet": 1.0}
        s, td = jvp_init(raw, zero, mask, cfg, **kw)
        jvp_run(s, td, mask, cfg, 6, "SSPRK2", 0.5, **kw)
        outs = []
        for sign in (1.0, -1.0):
            pp = with_params(1.0 + sign * eps, 0.0) if which == "d50" else with_params(1.0, sign * eps)
            b2, c2, m2, r2 = build(pp)
            st = b2.init_fn(r2, m2, c2)
            run_steps(st, m2, c2, "SSPRK2", 6, 0.5)
            outs.append(st.to_numpy())
        got = td.to_numpy()
        for f in ("h", "hu", "hv", "z_b", "G") if which == "d50" else ("h", "hu", "hv", "G"):
            fd = (outs[0][f] - outs[1][f]) / (2 * eps)
            assert np.max(np.abs(fd)) > 0, (which, f)
            assert rel_err(got[f], fd) <= tol, (which, f, rel_err(got[f], fd))


# ------------------------------------------------------------------ reverse mode
def inner(a, b, fields=("h", "hu", "hv", "z_b", "G")):
    A, B = a.to_numpy(), b.to_numpy()
    return float(sum(np.sum(A[f] * B[f]) for f in fields))


def random_adjoint(st, rng, fields=("h", "hu", "hv", "z_b", "G")):
    t = st.clone()
    for f in st.PLANES:
        getattr(t, f).zero_()
    for f in fields:
        getattr(t, f).copy_(torch.from_numpy(rng.standard_normal(st.shape)))
    return t


@pytest.mark.parametrize("scheme,layout,every", [("SSPRK2", "trans_x_refl_y", 32), ("SSPRK2", "influx_left", 3),
                                                 ("FE", "refl_all", 4), ("SSPRK2", "l_domain", 5)])
def test_adjoint_is_the_transpose_of_the_tangent(scheme, layout, every):
    """<abar_0, du_0> == <abar_N, J du_0>: the reverse mode (checkpointed, segments of
    `every` steps) against the tangent-linear run of the same 8 steps; both differentiate
    the same discrete map with the same branch choices, so they agree to rounding."""
    from pyexner_b200.tangent import jvp_run, vjp_run

    args = smooth_case(layout=layout)
    if layout == "l_domain":
        args[0]["z"][:6, -6:] = np.nan
    bundle, cfg, mask, st = setup(*args)
    rng = np.random.default_rng(17)
    du = tangent_state(st, rng, ("h", "hu", "hv", "z_b"))
    s, td = st.clone(), du.clone()
    jvp_run(s, td, mask, cfg, 8, scheme, 0.5)
    abar = random_adjoint(st, rng)
    rhs = inner(abar, td)
    a0 = vjp_run(st, abar.clone(), mask, cfg, 8, scheme, 0.5, checkpoint_every=every)
    lhs = inner(a0, du, ("h", "hu", "hv", "z_b"))
    assert abs(lhs - rhs) <= 1e-9 * max(abs(rhs), 1e-30), (lhs, rhs)


def test_bed_gradient_against_central_differences():
    """Gradient of J = sum (z + z_b - target)^2 after 10 SSPRK2 steps with respect to the
    bed of 12 random cells (through init), against central differences (eps 1e-6)."""
    from pyexner_b200 import BoundaryManager, RoeExnerState, create_solver_bundle, run_steps
    from pyexner_b200.cases import seds_matrix
    from pyexner_b200.tangent import vjp_init, vjp_run

    arrs, params, X, Y = smooth_case()
    bm = BoundaryManager(params, X, Y)
    raw = RoeExnerState.from_numpy(arrs, seds_matrix(params["erosion"]), torch.float64)
    bundle = create_solver_bundle("Roe Exner")
    cfg = bundle.config(raw, None, bm, 0.1, params)
    mask = bundle.mask_fn(raw, None, bm.boundary_mask)
    rng = np.random.default_rng(23)
    target = (arrs["z"] + arrs["z_b"]) + 0.001 * rng.standard_normal(arrs["h"].shape)

    def objective(st0_raw):
        st = bundle.init_fn(st0_raw, mask, cfg)
        run_steps(st, mask, cfg, "SSPRK2", 10, 0.5)
        s = st.to_numpy()
        return float(np.sum((s["z"] + s["z_b"] - target) ** 2)), st

    J0, stN = objective(raw)
    s = stN.to_numpy()
    abar = raw.clone()
    for f in raw.PLANES:
        getattr(abar, f).zero_()
    abar.z_b.copy_(torch.from_numpy(2 * (s["z"] + s["z_b"] - target)))
    st0 = bundle.init_fn(raw, mask, cfg)
    vjp_run(st0, abar, mask, cfg, 10, "SSPRK2", 0.5, checkpoint_every=4)
    vjp_init(raw, abar, mask, cfg)
    grad = abar.to_numpy()["z_b"]
    ny, nx = raw.shape
    cells = [(int(rng.integers(1, ny - 1)), int(rng.integers(1, nx - 1))) for _ in range(12)]
    eps = 1e-6
    for (r, c) in cells:
        vals = []
        for sign in (1.0, -1.0):
            p = raw.clone()
            p.z_b[r, c] += sign * eps
            vals.append(objective(p)[0])
        fd = (vals[0] - vals[1]) / (2 * eps)
        assert abs(grad[r, c] - fd) <= 1e-5 * max(abs(fd), 1e-8), ((r, c), grad[r, c], fd)


def test_torch_backward_through_the_function():
    """loss.backward() through RoeExnerSteps runs the adjoint kernels: the gradient equals
    the direct reverse-mode call (to 1e-12: the adjoint's atomic sums make the last bits
    depend on the order in which the GPU adds them)."""
    from pyexner_b200.tangent import RoeExnerSteps, StepsSpec, vjp_run

    bundle, cfg, mask, st = setup(*smooth_case())
    spec = StepsSpec(mask, cfg, st.seds, 4, "SSPRK2", 0.5)
    planes = [getattr(st, f).clone().requires_grad_(f in ("h", "hu", "hv", "z_b", "G")) for f in st.PLANES]
    out = RoeExnerSteps.apply(spec, *planes)
    zb_out = out[st.PLANES.index("z_b")]
    loss = (zb_out ** 2).sum() + out[0].sum()
    loss.backward()
    abar = st.clone()
    for f in st.PLANES:
        getattr(abar, f).zero_()
    abar.z_b.copy_(2 * zb_out.detach())
    abar.h.fill_(1.0)
    vjp_run(st, abar, mask, cfg, 4, "SSPRK2", 0.5)
    ref = abar.to_numpy()
    for k, f in enumerate(st.PLANES):
        if f in ("h", "hu", "hv", "z_b", "G"):
            assert rel_err(planes[k].grad.cpu().numpy(), ref[f]) <= 1e-12, f
