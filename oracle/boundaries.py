"""Ghost-cell boundary conditions restated in NumPy (oracle; test infrastructure only).

Follows PyExner src/PyExner/domain/boundary_registry.py and the handlers in
src/PyExner/domain/boundaries/.  Handlers are applied in YAML order; within one
handler every read happens before any write (a gather, then a scatter), and a later
handler overwrites an earlier one ("last writer wins" at corners).
"""
from __future__ import annotations

import numpy as np


def point_in_polygon(x, y, poly):
    """Even-odd ray casting (boundary_registry.py:19-44), vectorised over points."""
    xi, yi = poly[:, 0], poly[:, 1]
    xj, yj = np.roll(xi, 1), np.roll(yi, 1)
    x = x[:, None]
    y = y[:, None]
    crosses = (yi > y) != (yj > y)
    den = np.where(crosses, yj - yi, 1.0)
    tx = xi + (xj - xi) * (y - yi) / den
    hit = crosses & (x <= tx + 1e-8)
    return np.sum(hit, axis=1) % 2 == 1


def label_masks(X, Y, polygons):
    """One cell mask per boundary polygon, polygons zero-padded to a common vertex
    count as the reference does (boundary_registry.py:116-125)."""
    nv = max(len(p) for p in polygons)
    out = []
    for p in polygons:
        p = np.asarray(p, dtype=np.float64)
        p = np.pad(p, ((0, nv - p.shape[0]), (0, 0)))
        out.append(point_in_polygon(X.ravel(), Y.ravel(), p).reshape(X.shape))
    return out


def index_maps(mask, normal):
    """Boundary cells and their interior donors (boundary_registry.py:61-82).

    The donor is the cell one step against the outward normal in raster order:
    (row + round(ny), col - round(nx)), clipped to the array.
    """
    dx = -int(np.round(normal[0]))
    dy = int(np.round(normal[1]))
    b = np.argwhere(mask)
    i = b + np.array([dy, dx])
    ny, nx = mask.shape
    i = np.clip(i, 0, np.array([ny - 1, nx - 1]))
    return (b[:, 0], b[:, 1]), (i[:, 0], i[:, 1])


class Handler:
    def __init__(self, kind, mask, normal, values):
        self.kind = kind
        self.mask = mask
        self.normal = np.asarray(normal, dtype=np.float64)
        # the reference parses values into a float32 array (boundary_registry.py:107-110)
        self.values = np.asarray(values, dtype=np.float32)
        if kind == "Roe Exner ZeroMomentum":
            # a mask handler without index maps (boundary_registry.py:164-169): list its cells
            c = np.argwhere(mask)
            self.b = self.i = (c[:, 0], c[:, 1])
        else:
            self.b, self.i = index_maps(mask, normal)

    def apply(self, st, time=0.0):
        st = dict(st)
        by, bx = self.b
        iy, ix = self.i
        nx, ny = self.normal
        k = self.kind
        v = self.values
        if k == "Roe Exner Reflective":  # roeexner_reflective.py:17-63
            hu_i = st["hu"][iy, ix]
            hv_i = st["hv"][iy, ix]
            mom_n = hu_i * nx + hv_i * ny
            mom_t = -hu_i * ny + hv_i * nx
            mom_r = -mom_n
            new = {
                "h": st["h"][iy, ix],
                "z_b": st["z_b"][iy, ix],
                "n": st["n"][iy, ix],
                "G": st["G"][iy, ix],
                "hu": mom_r * nx - mom_t * ny,
                "hv": mom_r * ny + mom_t * nx,
            }
        elif k == "Roe Exner Transmissive":  # roeexner_transmissive.py:17-31
            new = {f: st[f][iy, ix] for f in ("h", "hu", "hv")}
        elif k == "Roe Exner TransmissiveBed":  # roeexner_transmissivebed.py:17-27
            new = {"z_b": st["z_b"][iy, ix]}
        elif k == "Roe Exner ConstantInflux":  # roeexner_constantinflux.py:18-48
            q, ux, uy = self.values[0], self.values[1], self.values[2]
            new = {"hu": np.float64(q * ux), "hv": np.float64(q * uy)}
        elif k == "Roe Reflective":  # roe_reflective.py:18-44
            new = {
                "h": st["h"][iy, ix],
                "z": st["z"][iy, ix],
                "n": st["n"][iy, ix],
                "hu": st["hu"][iy, ix] * (1 - 2 * nx * nx),
                "hv": st["hv"][iy, ix] * (1 - 2 * ny * ny),
            }
        elif k == "Roe Transmissive":  # roe_transmissive.py:17-43
            new = {f: st[f][iy, ix] for f in ("h", "z", "n", "hu", "hv")}
        elif k == "Roe Exner ConstantOutflux":  # roeexner_constantoutflux.py:18-59
            q, vx, vy = v[0], v[1], v[2]
            h_i = np.maximum(st["h"][iy, ix], 1e-8)
            u_i = st["hu"][iy, ix] / h_i
            v_i = st["hv"][iy, ix] / h_i
            un_i = u_i * vx + v_i * vy
            rp = un_i + 2.0 * np.sqrt(9.81 * h_i)
            h = h_i
            for _ in range(5):  # Newton on the outgoing Riemann invariant
                h = np.maximum(h, 1e-8)
                c = np.sqrt(9.81 * h)
                f = q / h + 2.0 * c - rp
                df = -q / (h * h) + 9.81 / np.maximum(c, 1e-8)
                h = np.maximum(h - f / df, 1e-8)
            new = {"h": h, "hu": np.float64(q * vx), "hv": np.float64(q * vy)}
        elif k in ("Roe Exner Berthon", "Roe Exner NormalFlowDepth"):
            # roeexner_berthon.py:19-56, roeexner_normalflowdepth.py:19-51 (float32 values)
            q, A, alpha, beta, gamma, x = v[0], v[1], v[2], v[3], v[4], v[5]
            u = np.power((alpha * x + beta) / A, np.float32(1.0 / 3.0))
            zb0 = -(u * (u * u) + 2.0 * 9.81 * q) / (2.0 * 9.81 * np.maximum(u, np.float32(1e-12))) + gamma
            zb = -alpha * np.float32(time) + zb0
            new = {"z_b": np.float64(zb)}
            if k == "Roe Exner NormalFlowDepth":
                new.update(h=np.float64(q / u), hu=st["hu"][iy, ix], hv=st["hv"][iy, ix])
        elif k == "Roe Exner SteepFall":  # roeexner_steepfall.py:17-26
            new = {"z_b": st["z_b"][iy, ix] - 1}
        elif k == "Roe Exner ZeroMomentum":  # roeexner_zeromomentum.py:16-31 (mask, no donors)
            m = self.mask
            hu_val = v[1] * self.normal[0]
            hv_val = v[1] * self.normal[1]
            st["hu"] = np.where(m, st["hu"] if np.isnan(hu_val) else hu_val, st["hu"])
            st["hv"] = np.where(m, st["hv"] if np.isnan(hv_val) else hv_val, st["hv"])
            return st
        else:
            raise KeyError(f"boundary type '{k}' is not on the oracle's path")
        for f, v in new.items():
            a = st[f].copy()
            a[by, bx] = v
            st[f] = a
        return st


class Boundaries:
    """``BoundaryManager`` (boundary_registry.py:84-187) for one rank."""

    def __init__(self, flux_scheme, specs, X, Y):
        polys = [specs[k]["polygon"] for k in specs]
        masks = label_masks(np.asarray(X), np.asarray(Y), polys)
        self.boundary_mask = np.any(np.stack(masks), axis=0)
        self.handlers = []
        for (name, spec), m in zip(specs.items(), masks):
            kind = flux_scheme + " " + spec["type"]
            vals = [np.nan if str(v).lower() == "nan" else float(v) for v in spec.get("values", [])]
            self.handlers.append(Handler(kind, m, spec["normal"], vals))

    def apply(self, st, time=0.0):
        for hd in self.handlers:
            st = hd.apply(st, time)
        return st


def roe_exner_mask(z, boundary_mask):
    """``get_mask`` on a single rank (roe_exner_solver.py:21-39)."""
    m = np.isnan(z)
    m[0, :] = True
    m[-1, :] = True
    m[:, 0] = True
    m[:, -1] = True
    m = np.where(boundary_mask, False, m)
    return np.stack([m, boundary_mask], axis=0)
