"""Seeded synthetic workloads (no dataset is involved; every input is generated).

* ``dambreak_roe``   plain Roe dam-break on the unit square: 256 x 256 cells
  (+ ring), dx = 1/256, h = 1 for x < 0.5 else 0.1, at rest, flat bed, Roe Reflective
  walls on the four sides (left, right, bottom, top), CFL 0.5, SSPRK2, 200 steps, float64.
* ``gaussian_bed``   Roe-Exner on an N x N grid (+ ring), dx = 0.01 m.  Total bed
  z_t = 0.05 * sum_{k<16} A_k exp(-|x - c_k|^2 / (2 s_k^2)) with c_k ~ U(domain),
  s_k ~ U(0.05, 0.3) L, A_k ~ U(-1, 1) (seed ``seed_bed``); rigid bed z = min(z_t) - 0.05
  (constant), erodible layer z_b = z_t - z; h = max(0, (0.3 - z_t) (1 + 0.02 U(-1, 1)))
  (seed ``seed_noise``), hu = 0.1 h, hv = 0, n = 0; MPM with one sediment
  (d = 1.61e-3 m, 2630 kg/m^3, porosity 0.42); Transmissive + TransmissiveBed in x,
  Reflective in y applied last (they win the corners).  N = 2048 is the 2000-step
  accuracy/throughput case, N = 8192 the 500-step bandwidth case.
"""
from __future__ import annotations

import numpy as np

from .boundaries import BoundaryManager, index_coords, ring_boundaries

SED_ONE = {"s1": dict(fraction=1.0, diameter=1.61e-3, density=2630.0, deposition_flux=0.0, erosion_flux=0.0)}


def seds_matrix(erosion):
    """7 x nsed matrix of src/PyExner/io/pnetcdf_reader.py:136-162 (theta_c = 0.047)."""
    grass = erosion["grass_factor"]
    if not isinstance(grass, str):
        return np.zeros((1, 1))
    rows = []
    for key in erosion["sediments"]:
        s = erosion["sediments"][key]
        rows.append([s["fraction"], s["diameter"], s["density"], s["deposition_flux"], s["erosion_flux"], 0.047,
                     erosion["bulk_porosity"]])
    return np.array(rows, dtype=np.float64).T


def dambreak_roe(n=256):
    ny = nx = n + 2
    dx = 1.0 / n
    xc = (np.arange(nx) - 0.5) * dx
    h = np.where(xc[None, :] < 0.5, 1.0, 0.1) * np.ones((ny, nx))
    z = np.zeros((ny, nx))
    arrs = dict(h=h, hu=np.zeros_like(h), hv=np.zeros_like(h), z=z, n=np.zeros_like(h))
    bspec = ring_boundaries(ny, nx, ["Reflective"], ["Reflective"], ["Reflective"], ["Reflective"])
    X, Y = index_coords(ny, nx)
    params = dict(flux_scheme="Roe", boundaries=bspec, cfl=0.5, integrator="SSPRK2")
    return dict(arrs=arrs, dx=dx, params=params, boundaries=BoundaryManager(params, X, Y), X=X, Y=Y)


def gaussian_bed_fields(n, dx=0.01, seed_bed=1, seed_noise=2, device=None, u0=0.1):
    """Planes of the Gaussian-bed case as float64 numpy arrays (ring included).

    With ``device`` set (e.g. "cuda") the bed sum is evaluated with torch on that device,
    which is what makes the 8192^2 case quick to build; the numbers are the same
    float64 expression either way.  ``u0`` is the initial velocity (hu = u0 h): the
    default 0.1 m/s keeps the Shields number near 1.5e-3, far below the threshold 0.047
    (no bedload at the start); 1 m/s gives about 0.15, bedload everywhere."""
    zt = gaussian_bed_total(n, n, dx, seed_bed, device)
    z = np.full(zt.shape, zt.min() - 0.05)
    zb = zt - z
    rn = np.random.default_rng(seed_noise)
    noise = rn.uniform(-1.0, 1.0, zt.shape)
    h = np.maximum(0.0, (0.3 - zt) * (1.0 + 0.02 * noise))
    return dict(h=h, hu=u0 * h, hv=np.zeros_like(h), z=z, z_b=zb, n=np.zeros_like(h), G=np.zeros_like(h))


def gaussian_bed_total(ny_phys, nx_phys, dx=0.01, seed_bed=1, device=None):
    """z_t = 0.05 sum_k A_k exp(-|x - c_k|^2 / (2 s_k^2)) on the (ny+2, nx+2) grid with
    ring: c_k ~ U(domain), s_k ~ U(0.05, 0.3) L with L = sqrt(Lx Ly) (the side of a square
    domain), A_k ~ U(-1, 1)."""
    ny, nx = ny_phys + 2, nx_phys + 2
    Lx, Ly = nx_phys * dx, ny_phys * dx
    L = float(np.sqrt(Lx * Ly))
    rb = np.random.default_rng(seed_bed)
    ck = rb.uniform(0.0, 1.0, (16, 2)) * np.array([Lx, Ly])
    sk = rb.uniform(0.05, 0.3, 16) * L
    ak = rb.uniform(-1.0, 1.0, 16)
    xc = (np.arange(nx) - 0.5) * dx
    yc = (ny - 1 - np.arange(ny) - 0.5) * dx
    if device is None:
        zt = np.zeros((ny, nx))
        for k in range(16):
            gx = np.exp(-((xc - ck[k, 0]) ** 2) / (2 * sk[k] ** 2))
            gy = np.exp(-((yc - ck[k, 1]) ** 2) / (2 * sk[k] ** 2))
            zt += ak[k] * np.outer(gy, gx)
        zt *= 0.05
    else:
        import torch

        tx = torch.tensor(xc, dtype=torch.float64, device=device)
        ty = torch.tensor(yc, dtype=torch.float64, device=device)
        acc = torch.zeros((ny, nx), dtype=torch.float64, device=device)
        for k in range(16):
            gx = torch.exp(-((tx - ck[k, 0]) ** 2) / (2 * sk[k] ** 2))
            gy = torch.exp(-((ty - ck[k, 1]) ** 2) / (2 * sk[k] ** 2))
            acc += ak[k] * torch.outer(gy, gx)
        zt = (0.05 * acc).cpu().numpy()
    return zt


def gaussian_bed(n, dx=0.01, seed_bed=1, seed_noise=2, device=None, u0=0.1):
    ny = nx = n + 2
    arrs = gaussian_bed_fields(n, dx, seed_bed, seed_noise, device, u0)
    erosion = dict(grass_factor="MPM", bulk_porosity=0.42, sediments=SED_ONE)
    bspec = ring_boundaries(ny, nx, ["Transmissive", "TransmissiveBed"], ["Transmissive", "TransmissiveBed"],
                            ["Reflective"], ["Reflective"])
    X, Y = index_coords(ny, nx)
    params = dict(flux_scheme="Roe Exner", integrator="SSPRK2", cfl=0.5, erosion=erosion, boundaries=bspec)
    return dict(arrs=arrs, seds=seds_matrix(erosion), dx=dx, params=params,
                boundaries=BoundaryManager(params, X, Y), X=X, Y=Y)


def adjoint_case(n=512, q_in=0.3, seed_initial=1, seed_target=2, dx=0.01):
    """Configuration 4: the Gaussian-bed generator at n x n (seed ``seed_initial``) started
    at 1 m/s, a ConstantInflux inlet of ``q_in`` m^2/s (values [q_in, 1, 0]) with
    TransmissiveBed on the left, Transmissive + TransmissiveBed on the right, Reflective in
    y (MPM, one sediment), and the target total bed z_t of the same generator with seed
    ``seed_target``.  Returns (arrs, params, X, Y, target)."""
    import copy

    ny = nx = n + 2
    arrs = gaussian_bed_fields(n, dx, seed_bed=seed_initial, u0=1.0)
    target = gaussian_bed_total(n, n, dx, seed_bed=seed_target)
    bspec = ring_boundaries(ny, nx, [("ConstantInflux", [q_in, 1.0, 0.0, 0.0]), "TransmissiveBed"],
                            ["Transmissive", "TransmissiveBed"], ["Reflective"], ["Reflective"])
    erosion = dict(grass_factor="MPM", bulk_porosity=0.42, sediments=copy.deepcopy(SED_ONE))
    params = dict(flux_scheme="Roe Exner", integrator="SSPRK2", cfl=0.5, erosion=erosion, boundaries=bspec)
    X, Y = index_coords(ny, nx)
    return arrs, params, X, Y, target


# ------------------------------------------------------------------ Berthon analytic case
BERTHON = dict(q=1.0, A=0.005, alpha=0.005, beta=0.005, gamma=1.0)


def berthon_exact(x, t, q=1.0, A=0.005, alpha=0.005, beta=0.005, gamma=1.0, g=9.81):
    """Analytic steady-flow / linearly eroding bed of Berthon et al. (the reference's
    tests/runtime/2D_const_flux/analyze_convergence.py:9-25): with a constant grass
    factor A, u = ((alpha x + beta) / A)^(1/3), h = q / u, hu = q and
    z_b = -alpha t - (u^3 + 2 g q) / (2 g u) + gamma, so that dz_b/dt = -alpha exactly."""
    u = ((alpha * x + beta) / A) ** (1.0 / 3.0)
    h = q / u
    zb = -alpha * t - (u**3 + 2 * g * q) / (2 * g * u) + gamma
    return h, q * np.ones_like(x), zb


def berthon_case(dh=0.1, end_time=10.0, out_freq=1.0, integrator="Forward Euler"):
    """Input of the reference's 2D_const_flux case (tests/runtime/2D_const_flux/
    2D_build_num_sol.py:8-56 and input.yaml): the analytic state at t = 0 on
    x in [0, 7], y in [0, 1] (file rows from y = 1 down to 0) with spacing dh, and the
    run parameters: constant grass factor 0.005, ConstantInflux + Berthon bed at the
    inlet, NormalFlowDepth at the outlet, reflective walls, CFL 0.5.

    Returns (x, y, fields, params): file coordinates, float64 planes and the YAML dict
    (without input_file / output_file)."""
    c = BERTHON
    x = np.arange(0.0, 7.0 + dh, dh)
    y = np.arange(1.0, 0.0 - dh, -dh)
    X, _ = np.meshgrid(x, y, indexing="xy")
    h, hu, zb = berthon_exact(X, 0.0, **c)
    zeros = np.zeros_like(h)
    fields = dict(h=h, hu=hu, hv=zeros, z_b=zb, z=zeros, n=zeros)
    vals = [c["q"], c["A"], c["alpha"], c["beta"], c["gamma"]]
    params = dict(
        end_time=end_time, out_freq=out_freq, cfl=0.5, flux_scheme="Roe Exner", integrator=integrator,
        parNx=1, parNy=1, erosion=dict(grass_factor=0.005),
        boundaries=dict(
            inlet_flux=dict(type="ConstantInflux", polygon=[[0.0, 0.0], [0.05, 0.0], [0.05, 1.0], [0.0, 1.0]],
                            values=[1.0, 1.0, 0.0], normal=[-1.0, 0.0]),
            inlet_bed=dict(type="Berthon", polygon=[[0.0, 0.0], [0.05, 0.0], [0.05, 1.0], [0.0, 1.0]],
                           values=vals + [0.025], normal=[-1.0, 0.0]),
            outlet_bed=dict(type="NormalFlowDepth", polygon=[[6.95, 0.0], [7.05, 0.0], [7.05, 1.05], [6.95, 1.05]],
                            values=vals + [6.975], normal=[1.0, 0.0]),
            bottom=dict(type="Reflective", polygon=[[0.0, -0.05], [7.05, -0.05], [7.05, 0.05], [0.0, 0.05]],
                        values=[0, 0, 0, 0], normal=[0.0, -1.0]),
            top=dict(type="Reflective", polygon=[[0.0, 1.05], [7.05, 1.05], [7.05, 0.95], [0.0, 0.95]],
                     values=[0, 0, 0, 0], normal=[0.0, 1.0]),
        ),
    )
    return x, y, fields, params


# ------------------------------------------------------------------ ragged ensemble
def ensemble_fields(ny_phys, nx_phys, step_height, dx=0.01, seed_bed=1):
    """One member of the ragged dam-break ensemble: the Gaussian-sum bed of
    ``gaussian_bed_total`` on an ny x nx grid (split into a constant rigid bed 5 cm below
    its minimum and the erodible layer above it), water at rest at
    h = max(0, 0.3 - z_t) + H [x < Lx / 2]."""
    zt = gaussian_bed_total(ny_phys, nx_phys, dx, seed_bed)
    z = np.full(zt.shape, zt.min() - 0.05)
    zb = zt - z
    xc = (np.arange(nx_phys + 2) - 0.5) * dx
    h = np.maximum(0.0, 0.3 - zt) + step_height * (xc[None, :] < 0.5 * nx_phys * dx)
    zeros = np.zeros_like(h)
    return dict(h=h, hu=zeros.copy(), hv=zeros.copy(), z=z, z_b=zb, n=zeros.copy(), G=zeros.copy())


def ensemble_case(count=64, seed=0, sides=(128, 1024), heights=(0.2, 1.0), dx=0.01):
    """The ragged ensemble workload: ``count`` Roe-Exner dam breaks whose grid sides are
    drawn independently from U{sides} (seeded, non-square allowed), each with its own
    Gaussian-sum bed (seed ``1000 * seed + k``) and its own step height H ~ U(heights);
    MPM with one sediment, Transmissive + TransmissiveBed in x, Reflective in y.

    Returns (members, erosion): ``members`` holds per member ``arrs`` (float64 planes with
    the ring), ``shape``, ``height``, ``dx`` and the YAML-style ``params``."""
    rs = np.random.default_rng(seed)
    erosion = dict(grass_factor="MPM", bulk_porosity=0.42, sediments=SED_ONE)
    members = []
    for k in range(count):
        nyp, nxp = (int(v) for v in rs.integers(sides[0], sides[1] + 1, 2))
        H = float(rs.uniform(heights[0], heights[1]))
        arrs = ensemble_fields(nyp, nxp, H, dx, seed_bed=1000 * seed + k)
        ny, nx = nyp + 2, nxp + 2
        bspec = ring_boundaries(ny, nx, ["Transmissive", "TransmissiveBed"], ["Transmissive", "TransmissiveBed"],
                                ["Reflective"], ["Reflective"])
        params = dict(flux_scheme="Roe Exner", integrator="SSPRK2", cfl=0.5, erosion=erosion, boundaries=bspec)
        members.append(dict(arrs=arrs, shape=(ny, nx), height=H, dx=dx, params=params))
    return members, erosion
