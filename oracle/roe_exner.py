"""Roe-Exner step restated in NumPy float64 (oracle; test infrastructure only).

Every function cites the PyExner source it follows (paths relative to the PyExner
project root, ``src/`` = ``src/PyExner/``).  Expressions keep the reference's operation
order so that float64 results agree with the reference's to the last bit where numpy
is the arithmetic.

A state is a dict with the planes ``h, hu, hv, z, z_b, n, n_b, G`` (shape (Ny, Nx),
ring included) and ``seds`` (7 x nsed: fraction, d50, density, k_d, k_e, theta_c,
porosity; src/io/pnetcdf_reader.py:136-158).  ``mask`` is the (2, Ny, Nx) bool stack of
src/solvers/roe_exner_solver.py:21-39: mask[0] = nodata (NaN bed or uncovered ring),
mask[1] = boundary-condition cells.
"""
from __future__ import annotations

import numpy as np

# src/utils/constants.py:23-33
G_ACC = 9.81
DRY_TOL = 1e-4
SED_TOL = 1e-5
VEL_TOL = 1e-6
DT_FLOOR = 1e-6  # src/solvers/roe_exner_solver.py:121

STATE_FIELDS = ("h", "hu", "hv", "z", "z_b", "n", "n_b", "G")

# Face orientations: x-faces join (r, c)|(r, c+1) with normal (1, 0); y-faces join
# (r, c)|(r+1, c) with normal (0, -1) (src/solvers/kernels/roe_exner.py:576-577).
NORMAL_X = (1, 0)
NORMAL_Y = (0, -1)


def _rotate(u, v, normal):
    """Normal / tangential velocity for an axis normal.

    The reference forms ``u*nx + v*ny`` and ``-u*ny + v*nx`` with integer normals
    (roe_exner.py:329-333); for (1,0) and (0,-1) those sums are exact, so the
    components are (u, v) and (-v, u).
    """
    if normal == NORMAL_X:
        return u, v
    return -v, u


def _rotate_back(c0, c1, c2, normal):
    """Tk_inv back-rotation (roe_exner.py:526-531), exact for axis normals."""
    if normal == NORMAL_X:
        return c0, c1, c2
    return c0, c2, -c1


def roe_face(si, sj, normal, dx):
    """Roe-Exner hydrodynamic fluctuations of one face set.

    Follows src/solvers/kernels/roe_exner.py:312-533 (``roe_solver``).  ``si``/``sj`` are
    tuples (h, hu, hv, z_b, z, n_b) of the two cells.  Returns (upwP, upwM), each a
    tuple of 3 arrays in (h, hu, hv) order: upwP goes to cell j, upwM to cell i.
    """
    hi, hui, hvi, z_bi, zi, ni = si
    hj, huj, hvj, z_bj, zj, nj = sj
    hi = np.maximum(hi, DRY_TOL)
    hj = np.maximum(hj, DRY_TOL)
    with np.errstate(all="ignore"):
        ui = np.where(hi > DRY_TOL, hui / hi, 0.0)
        vi = np.where(hi > DRY_TOL, hvi / hi, 0.0)
        uj = np.where(hj > DRY_TOL, huj / hj, 0.0)
        vj = np.where(hj > DRY_TOL, hvj / hj, 0.0)
        uhi, vhi = _rotate(ui, vi, normal)
        uhj, vhj = _rotate(uj, vj, normal)
        sqi = np.sqrt(hi)
        sqj = np.sqrt(hj)
        den = sqi + sqj
        ht = 0.5 * (hi + hj)
        ct = np.sqrt(G_ACC * ht)
        ut = (uhi * sqi + uhj * sqj) / den
        vt = (vhi * sqi + vhj * sqj) / den
        l1r = ut - ct
        l2 = ut
        l3r = ut + ct
        # Harten-Hyman entropy fix (roe_exner.py:357-371); VEL_TOL only in the lambda_3 branch
        ei = uhi - np.sqrt(G_ACC * hi)
        ej = uhj - np.sqrt(G_ACC * hj)
        m1 = (ei < 0.0) & (ej > 0.0)
        lE1 = np.where(m1, l1r - ei * (ej - l1r) / (ej - ei), 0.0)
        l1 = np.where(m1, ei * (ej - l1r) / (ej - ei), l1r)
        ei = uhi + np.sqrt(G_ACC * hi)
        ej = uhj + np.sqrt(G_ACC * hj)
        m3 = (ei < 0.0) & (ej > 0.0)
        lE3 = np.where(m3, l3r - ej * (l3r - ei) / (ej - ei), 0.0)
        l3 = np.where(m3, ej * (l3r - ei) / ((ej - ei) + VEL_TOL), l3r)
        # wave strengths with the unfixed speeds (roe_exner.py:399-412)
        dh = hj - hi
        dhu = hj * uhj - hi * uhi
        dhv = hj * vhj - hi * vhi
        den2 = -2.0 * ct
        a1 = (-l3r * dh + dhu) / den2
        a2 = (-vt * dh + dhv) / ct
        a3 = (l1r * dh - dhu) / den2
        # bed step with the sediment floor (roe_exner.py:421-432)
        z_bi = np.where(z_bi > SED_TOL, z_bi, SED_TOL * 0.01)
        z_bj = np.where(z_bj > SED_TOL, z_bj, SED_TOL * 0.01)
        dz = (zj + z_bj) - (zi + z_bi)
        thrust = -G_ACC * ht * dz
        # Manning friction (roe_exner.py:455-457)
        nt = 0.5 * (ni + nj)
        sf = (nt**2 * np.sqrt(ut**2 + vt**2) * ut) / (np.maximum(DRY_TOL, ht ** (4 / 3)))
        tau = G_ACC * ht * sf * dx
        b1 = (thrust - tau) / den2
        b3 = -b1
        # The dry masks mask_1/mask_2 (roe_exner.py:480-481) test the clamped depth
        # against DRY_TOL and are never true; the sign split alone remains.
        lam = (l1, l2, l3)
        alp = (a1, a2, a3)
        bet = (b1, 0.0, b3)
        zeros = np.zeros_like(ut)
        P = ((1.0, l1, vt), (zeros, zeros, ct), (1.0, l3, vt))  # columns of P (roe_exner.py:379-383)
        pos = [zeros, zeros, zeros]
        neg = [zeros, zeros, zeros]
        for k in range(3):
            w = lam[k] * alp[k] - bet[k]
            for r in range(3):
                f = w * P[k][r]
                pos[r] = pos[r] + np.where(lam[k] > 0.0, f, 0.0)
                neg[r] = neg[r] + np.where(lam[k] <= 0.0, f, 0.0)
        lamE = (lE1, zeros, lE3)
        for k in range(3):
            for r in range(3):
                f = lamE[k] * alp[k] * P[k][r]
                pos[r] = pos[r] + np.where(lamE[k] > 0.0, f, 0.0)
                neg[r] = neg[r] + np.where(lamE[k] <= 0.0, f, 0.0)
    return _rotate_back(*pos, normal), _rotate_back(*neg, normal)


def _pairs(arrs, axis):
    if axis == 1:
        return tuple(a[:, :-1] for a in arrs), tuple(a[:, 1:] for a in arrs)
    return tuple(a[:-1, :] for a in arrs), tuple(a[1:, :] for a in arrs)


def face_active(h, mask0, axis):
    """Either side wet and neither side nodata (roe_exner.py:581-588)."""
    (hi,), (hj,) = _pairs((h,), axis)
    (mi,), (mj,) = _pairs((mask0,), axis)
    return ((hi > DRY_TOL) | (hj > DRY_TOL)) & ~(mi | mj)


def hydro_update(st, dt, dx, mask):
    """``roe_solve_2D`` (roe_exner.py:535-612): returns new (h, hu, hv) on all cells."""
    arrs = (st["h"], st["hu"], st["hv"], st["z_b"], st["z"], st["n_b"])
    ny, nx = st["h"].shape
    flux = [np.zeros((ny, nx)) for _ in range(3)]
    res = {}
    for axis, normal in ((1, NORMAL_X), (0, NORMAL_Y)):
        si, sj = _pairs(arrs, axis)
        P, M = roe_face(si, sj, normal, dx)
        act = face_active(st["h"], mask[0], axis)
        res[axis] = ([np.where(act, p, 0.0) for p in P], [np.where(act, m, 0.0) for m in M])
    # scatter order of roe_exner.py:597-602: x upwM, x upwP, y upwM, y upwP
    for r in range(3):
        flux[r][:, :-1] += res[1][1][r]
        flux[r][:, 1:] += res[1][0][r]
        flux[r][:-1, :] += res[0][1][r]
        flux[r][1:, :] += res[0][0][r]
    return (st["h"] - dt * flux[0] / dx, st["hu"] - dt * flux[1] / dx, st["hv"] - dt * flux[2] / dx)


def momentum_corrections(h, hu, hv, z, z_b, mask0):
    """Interior momentum zeroing (roe_exner.py:14-62)."""
    hu = hu.copy()
    hv = hv.copy()
    C = (slice(1, -1), slice(1, -1))
    W = (slice(1, -1), slice(0, -2))
    E = (slice(1, -1), slice(2, None))
    N = (slice(0, -2), slice(1, -1))
    S = (slice(2, None), slice(1, -1))
    ztot = z + z_b
    eta = h[C] + ztot[C]
    stop_u = ((eta < ztot[E]) & (h[E] < DRY_TOL)) | ((eta < ztot[W]) & (h[W] < DRY_TOL)) | mask0[E] | mask0[W]
    stop_v = ((eta < ztot[N]) & (h[N] < DRY_TOL)) | ((eta < ztot[S]) & (h[S] < DRY_TOL)) | mask0[N] | mask0[S]
    active = (h[C] > DRY_TOL) & ~mask0[C]
    hu[C] = np.where(active & ~stop_u, hu[C], 0.0)
    hv[C] = np.where(active & ~stop_v, hv[C], 0.0)
    return hu, hv


def compute_n(n, z_b, seds):
    """Manning of the erodible layer (roe_exner.py:64-73)."""
    frac = seds[0][:, None, None]
    d50 = seds[1][:, None, None]
    d50 = np.mean(d50 * frac, axis=0)
    n_p = d50 ** (1 / 6) / 21.1
    return np.where(z_b > SED_TOL, n_p, n)


def compute_G_mpm(h, hu, hv, seds, mask0):
    """Meyer-Peter & Mueller grass factor (roe_exner.py:85-130)."""
    h = np.maximum(h, DRY_TOL)
    with np.errstate(all="ignore"):
        u = hu / h
        v = hv / h
        vel2 = u**2 + v**2
        frac, d50, density, k_d, k_e, theta_c, porosity = seds
        s = density / 1000.0
        n_p = d50 ** (1 / 6) / 21.1
        frac = frac[:, None, None]
        d50 = d50[:, None, None]
        s = s[:, None, None]
        n_p = n_p[:, None, None]
        theta_c = theta_c[:, None, None]
        theta = (n_p**2 * vel2) / ((s - 1.0) * d50 * np.cbrt(h))
        theta = np.maximum(theta, 0.0)
        dtheta = np.maximum(theta - theta_c, 0.0)
        sqrt_h = np.sqrt(h)
        # n_p**3 and b**3 below are jax integer_pow: repeated multiplication, not pow()
        g1 = n_p * (n_p * n_p) * np.sqrt(G_ACC) / ((s - 1.0) * sqrt_h)
        g2 = 8.0 * np.sqrt(dtheta) / (theta**1.5 + 1e-5)
        G = np.sum(frac * g1 * g2 * dtheta, axis=0)
        G = G / (1.0 - porosity.mean())
    G = np.where(mask0, 0.0, G)
    return np.where(h > DRY_TOL, G, 0.0)


def compute_G_const(h, G_in, mask0):
    """Constant grass factor pass-through (roe_exner.py:136-140)."""
    G = np.where(mask0, 0.0, G_in)
    return np.where(h > DRY_TOL, G, 0.0)


def compute_G(st, mask0, mpm):
    if mpm:
        return compute_G_mpm(st["h"], st["hu"], st["hv"], st["seds"], mask0)
    return compute_G_const(st["h"], st["G"], mask0)


def exner_face(si, sj, normal):
    """Upwind bedload flux of one face set (roe_exner.py:614-663, ``exner_solver``).

    ``si``/``sj`` are (h, hu, hv, z_b, z, G).
    """
    hi, hui, hvi, z_bi, zi, gi = si
    hj, huj, hvj, z_bj, zj, gj = sj
    hi = np.where(hi > DRY_TOL, hi, DRY_TOL * 0.01)
    hj = np.where(hj > DRY_TOL, hj, DRY_TOL * 0.01)
    z_bi = np.where(z_bi > SED_TOL, z_bi, SED_TOL * 0.01)
    z_bj = np.where(z_bj > SED_TOL, z_bj, SED_TOL * 0.01)
    with np.errstate(all="ignore"):
        sqi = np.sqrt(hi)
        sqj = np.sqrt(hj)
        ui = np.where(hi > DRY_TOL, hui / hi, 0.0)
        vi = np.where(hi > DRY_TOL, hvi / hi, 0.0)
        uj = np.where(hj > DRY_TOL, huj / hj, 0.0)
        vj = np.where(hj > DRY_TOL, hvj / hj, 0.0)
        uhi, _ = _rotate(ui, vi, normal)
        uhj, _ = _rotate(uj, vj, normal)
        ut = (uhi * sqi + uhj * sqj) / (sqi + sqj)
        umi = ui**2 + vi**2
        umj = uj**2 + vj**2
        qi = gi * umi * uhi
        qj = gj * umj * uhj
        gt = 0.5 * (gi + gj)
        dz = z_bj - z_bi
        dq = gt * umj * uhj - gt * umi * uhi
        lam4 = np.where(np.abs(dz) > SED_TOL, dq / dz, ut)
        qbi = qi + (gt - gi) * umi * uhi
        qbj = qj + (gt - gj) * umj * uhj
    return np.where(lam4 >= 0, qbi, qbj)


def exner_update(st, dt, dx, mask0):
    """``exner_solve_2D`` (roe_exner.py:665-717): new z_b on all cells."""
    arrs = (st["h"], st["hu"], st["hv"], st["z_b"], st["z"], st["G"])
    ny, nx = st["h"].shape
    F = {}
    for axis, normal in ((1, NORMAL_X), (0, NORMAL_Y)):
        si, sj = _pairs(arrs, axis)
        f = exner_face(si, sj, normal)
        (mi,), (mj,) = _pairs((mask0,), axis)
        stop = (mi | mj) | ((si[3] < SED_TOL) & (sj[3] < SED_TOL))
        depth = (si[0] > DRY_TOL) | (sj[0] > DRY_TOL)
        F[axis] = np.where(depth & ~stop, f, 0.0)
    flux = np.zeros((ny, nx))
    flux[:, 1:] += -F[1]
    flux[:, :-1] += F[1]
    flux[1:, :] += -F[0]
    flux[:-1, :] += F[0]
    return st["z_b"] - dt * flux / dx


def _lambda_cubic(ut, at, ct):
    """Extreme roots of the coupled bed/flow cubic (roe_exner.py:163-209, ``_get_lambda``).

    Trigonometric Cardano on -l^3 - 2u l^2 + ((1+a)c^2 - u^2) l - c^2 a u = 0, with the
    linear speeds u -/+ c when a < 1e-5.
    """
    a = -1
    b = -2 * ut
    c = (1 + at) * ct**2 - ut**2
    d = -ct**2 * at * ut
    with np.errstate(all="ignore"):
        p = (3 * a * c - b**2) / (3 * a**2)
        q = (2 * (b * (b * b)) - 9 * a * b * c + 27 * a**2 * d) / (27 * a**3)
        cos_t = np.clip((3 * q) / (2 * p) * np.sqrt(-3 / p), -1.0, 1.0)
        theta = np.arccos(cos_t)
        sq = 2 * np.sqrt(-p / 3)
        shift = -b / (3 * a)
        lmax = sq * np.cos(theta / 3) + shift
        lmin = sq * np.cos((theta + 2 * np.pi) / 3) + shift
    small = at < 1e-5
    return np.where(small, ut - ct, lmin), np.where(small, ut + ct, lmax)


def dt_face(si, sj, normal, dx):
    """Per-face stable step (roe_exner.py:211-255, ``compute_dt``). si = (h, hu, hv, z, G)."""
    hi, hui, hvi, zi, gi = si
    hj, huj, hvj, zj, gj = sj
    hi = np.maximum(hi, DRY_TOL)
    hj = np.maximum(hj, DRY_TOL)
    with np.errstate(all="ignore"):
        sqi = np.sqrt(hi)
        sqj = np.sqrt(hj)
        den = sqi + sqj
        ui = hui / hi
        vi = hvi / hi
        uj = huj / hj
        vj = hvj / hj
        uhi, vhi = _rotate(ui, vi, normal)
        uhj, vhj = _rotate(uj, vj, normal)
        ht = 0.5 * (hi + hj)
        ut = (uhi * sqi + uhj * sqj) / den
        ct = np.sqrt(G_ACC * ht)
        gt = 0.5 * (gi + gj)
        at = gt * (uhi**2 + uhi * uhj + uhj**2 + vhi * vhj) / (sqi * sqj)
        l1 = ut - ct
        l3 = ut + ct
        lmin, lmax = _lambda_cubic(ut, at, ct)
        roe_speed = np.maximum(np.abs(lmin), np.abs(lmax))
        swe_speed = np.maximum(np.abs(l1), np.abs(l3))
        return np.where(roe_speed < VEL_TOL, dx / swe_speed, dx / roe_speed)


def compute_dt_2D(st, dx, mask0):
    """Minimum face step over active faces, ring faces included (roe_exner.py:257-310)."""
    arrs = (st["h"], st["hu"], st["hv"], st["z"], st["G"])
    out = []
    for axis, normal in ((1, NORMAL_X), (0, NORMAL_Y)):
        si, sj = _pairs(arrs, axis)
        d = dt_face(si, sj, normal, dx)
        act = face_active(st["h"], mask0, axis)
        out.append(np.where(act, d, np.inf).min())
    return np.minimum(out[0], out[1])


def compute_dt(st, cfl, dx, mask0):
    """``compute_dt_roeexner`` on one rank (roe_exner_solver.py:118-122)."""
    return np.maximum(cfl * compute_dt_2D(st, dx, mask0), DT_FLOOR)


def init(st, mask, bcs, mpm):
    """``init_fn_roeexner`` on one rank (roe_exner_solver.py:58-78)."""
    st = dict(st)
    if mpm:
        st["n_b"] = compute_n(st["n"], st["z_b"], st["seds"])
    else:
        st["n_b"] = st["n"].copy()
    st["G"] = compute_G(st, mask[0], mpm)
    return bcs.apply(st)


def stage(st, dt, dx, mask, bcs, mpm, time=0.0):
    """``step_fn_roeexner`` on one rank (roe_exner_solver.py:80-116).

    hydro (a5) -> momentum corrections (a6) -> BCs (a7) -> G (a8) -> Exner (a9) -> BCs.
    ``n_b`` stays at its init value: the reference recomputes it and then discards the
    result (roe_exner_solver.py:112-113).
    """
    st = dict(st)
    h, hu, hv = hydro_update(st, dt, dx, mask)
    hu, hv = momentum_corrections(h, hu, hv, st["z"], st["z_b"], mask[0])
    st.update(h=h, hu=hu, hv=hv)
    st = bcs.apply(st, time)
    st["G"] = compute_G(st, mask[0], mpm)
    st["z_b"] = exner_update(st, dt, dx, mask[0])
    return bcs.apply(st, time)


def hydro_and_corrections(st, dt, dx, mask):
    """The first two sub-phases of a stage, exposed for finer-grained parity checks."""
    h, hu, hv = hydro_update(st, dt, dx, mask)
    hu_c, hv_c = momentum_corrections(h, hu, hv, st["z"], st["z_b"], mask[0])
    return h, hu, hv, hu_c, hv_c
