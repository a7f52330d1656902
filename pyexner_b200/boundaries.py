"""Ghost-cell boundary set-up (host side, off the clock).

Mirrors PyExner's ``BoundaryManager`` (src/PyExner/domain/boundary_registry.py:84-187):
each YAML ``boundaries`` entry names a polygon, a type, an outward normal and values;
the polygon selects cells by even-odd ray casting on the cell centres (:19-59) and
every selected cell takes its donor one step against the normal (:61-82).  The handler
list is handed to the C ABI in YAML order; the library resolves it into per-ring-cell
recipes that the fused stage kernel applies in registers, or applies the handlers one
after another on the general stage path.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


def point_in_polygon(x, y, poly):
    """Even-odd test of many points against one polygon (boundary_registry.py:19-44)."""
    xi, yi = poly[:, 0], poly[:, 1]
    xj, yj = np.roll(xi, 1), np.roll(yi, 1)
    x = x[:, None]
    y = y[:, None]
    crosses = (yi > y) != (yj > y)
    den = np.where(crosses, yj - yi, 1.0)
    tx = xi + (xj - xi) * (y - yi) / den
    return np.sum(crosses & (x <= tx + 1e-8), axis=1) % 2 == 1


def label_masks(X, Y, polygons):
    """One mask per polygon; polygons are zero-padded to a common vertex count as in
    boundary_registry.py:116-125."""
    nv = max(len(p) for p in polygons)
    out = []
    for p in polygons:
        p = np.asarray(p, dtype=np.float64)
        p = np.pad(p, ((0, nv - p.shape[0]), (0, 0)))
        out.append(point_in_polygon(np.ravel(X), np.ravel(Y), p).reshape(np.shape(X)))
    return out


def index_maps(mask, normal):
    """(boundary cells, donor cells) as (rows, cols) pairs (boundary_registry.py:61-82)."""
    b = np.argwhere(mask)
    return donor_maps((b[:, 0], b[:, 1]), normal, mask.shape)


def donor_maps(cells, normal, shape):
    """Donors of raster-ordered boundary cells: one step against the normal,
    (row + round(ny), col - round(nx)), clipped to the array (boundary_registry.py:61-82)."""
    dx = -int(np.round(normal[0]))
    dy = int(np.round(normal[1]))
    by, bx = cells
    ny, nx = shape
    return (by, bx), (np.clip(by + dy, 0, ny - 1), np.clip(bx + dx, 0, nx - 1))


def label_cells_device(X, Y, polygons):
    """Raster-ordered (rows, cols) of the cells inside each polygon, labelled on the GPU
    (``pxb_label_polygons``) with the host test's arithmetic.  X, Y must be a meshgrid
    (X constant down columns, Y constant along rows)."""
    X = np.asarray(X, dtype=np.float64)
    Y = np.asarray(Y, dtype=np.float64)
    ny, nx = X.shape
    xc = np.ascontiguousarray(X[0, :])
    yc = np.ascontiguousarray(Y[:, 0])
    if not (np.array_equal(X, np.broadcast_to(xc, X.shape)) and np.array_equal(Y, np.broadcast_to(yc[:, None], Y.shape))):
        raise ValueError("device labelling needs meshgrid coordinates")
    nv = max(len(p) for p in polygons)
    verts = np.zeros((len(polygons), nv, 2))
    for k, p in enumerate(polygons):
        p = np.asarray(p, dtype=np.float64)
        verts[k, : p.shape[0]] = p
    verts = np.ascontiguousarray(verts)
    counts = np.zeros(len(polygons), dtype=np.int64)
    args = (ny, nx, xc.ctypes.data, yc.ctypes.data, verts.ctypes.data, len(polygons), nv, counts.ctypes.data)
    _lib.call("pxb_label_polygons", *args, None, 0, None)
    cells = np.empty(max(1, int(counts.sum())), dtype=np.int64)
    _lib.call("pxb_label_polygons", *args, cells.ctypes.data, int(cells.size), None)
    out, o = [], 0
    for n in counts:
        idx = cells[o:o + n]
        out.append((idx // nx, idx % nx))
        o += n
    return out


class BoundaryManager:
    """Boundary handlers of one run, in YAML order.

    ``setup``: "host" labels the cells with NumPy, "device" on the GPU
    (``pxb_label_polygons``, for large grids), "auto" picks the device above 4M cells
    when a GPU is present.  Both give the same cells."""

    def __init__(self, params, X, Y, setup="auto"):
        self.flux_scheme = params["flux_scheme"]
        self.boundary_specs = params.get("boundaries") or {}
        self.names = list(self.boundary_specs)
        X = np.asarray(X)
        Y = np.asarray(Y)
        self.shape = X.shape
        self.handlers = []
        if not self.names:
            self.boundary_mask = np.zeros(self.shape, bool)
            return
        polys = [self.boundary_specs[k]["polygon"] for k in self.names]
        if setup == "auto":
            setup = "host"
            if X.size > (1 << 22):
                import torch

                if torch.cuda.is_available():
                    setup = "device"
        if setup == "device":
            cell_lists = label_cells_device(X, Y, polys)
        else:
            cell_lists = []
            for m in label_masks(X, Y, polys):
                b = np.argwhere(m)
                cell_lists.append((b[:, 0], b[:, 1]))
        self.boundary_mask = np.zeros(self.shape, bool)
        for by, bx in cell_lists:
            self.boundary_mask[by, bx] = True
        for name, cl in zip(self.names, cell_lists):
            spec = self.boundary_specs[name]
            kind = self.flux_scheme + " " + spec["type"]
            if kind not in _lib.BC_KINDS:
                raise KeyError(f"[BoundaryManager] Unknown boundary '{kind}'. Available options: {list(_lib.BC_KINDS)}")
            vals = np.array([np.nan if str(v).lower() == "nan" else float(v) for v in spec.get("values", [])],
                            dtype=np.float32)
            normal = [float(v) for v in spec["normal"]]
            if kind == "Roe Exner ZeroMomentum":
                # mask handler (roeexner_zeromomentum.py:16-31): every mask cell is its own donor
                (by, bx), (iy, ix) = cl, cl
            else:
                (by, bx), (iy, ix) = donor_maps(cl, normal, self.shape)
            hu_c = hv_c = 0.0
            if kind == "Roe Exner ConstantInflux":
                # float32 values as parsed by boundary_registry.py:107-110, product in float32
                hu_c = float(np.float32(vals[0]) * np.float32(vals[1]))
                hv_c = float(np.float32(vals[0]) * np.float32(vals[2]))
            self.handlers.append(dict(name=name, kind=kind, normal=normal, values=vals,
                                      cells=(by, bx), donors=(iy, ix), hu_const=hu_c, hv_const=hv_c))

    def c_array(self, pitch):
        """ctypes array of ``pxb_bc_handler`` (flat row*pitch+col indices); the index
        arrays are kept alive on the returned object."""
        n = len(self.handlers)
        arr = (_lib.BcHandler * max(1, n))()
        keep = []
        for k, hd in enumerate(self.handlers):
            by, bx = hd["cells"]
            iy, ix = hd["donors"]
            cells = np.ascontiguousarray(by.astype(np.int64) * pitch + bx, dtype=np.int64)
            donors = np.ascontiguousarray(iy.astype(np.int64) * pitch + ix, dtype=np.int64)
            keep += [cells, donors]
            arr[k].kind = _lib.BC_KINDS[hd["kind"]]
            arr[k].count = len(cells)
            arr[k].cells = cells.ctypes.data_as(ctypes.c_void_p)
            arr[k].donors = donors.ctypes.data_as(ctypes.c_void_p)
            arr[k].nx, arr[k].ny = hd["normal"]
            arr[k].hu_const = hd["hu_const"]
            arr[k].hv_const = hd["hv_const"]
            vals = hd["values"][:8]
            for j, v in enumerate(vals):
                arr[k].values[j] = float(v)  # float32 values, NaN kept
        arr._keep = keep
        return arr, n


def roe_exner_mask(z, boundary_mask):
    """``get_mask`` of the "Roe Exner" bundle on one rank (roe_exner_solver.py:21-39):
    mask[0] = NaN bed or outer ring, minus boundary cells; mask[1] = boundary cells."""
    m = np.isnan(np.asarray(z))
    m[0, :] = True
    m[-1, :] = True
    m[:, 0] = True
    m[:, -1] = True
    m = np.where(boundary_mask, False, m)
    return np.stack([m, boundary_mask], axis=0)


# ------------------------------------------------------------------ ring layouts
def _rect(x0, x1, y0, y1):
    return [[x0, y0], [x1, y0], [x1, y1], [x0, y1]]


def ring_boundaries(ny, nx, west, east, south, north):
    """YAML-style ``boundaries`` for the four sides of an index-space grid whose cell
    centres are X = column, Y = ny - 1 - row.  Each side is a list of handler types;
    sides are emitted west, east, south, north (later entries win the corners)."""
    polys = {
        "west": (_rect(-0.5, 0.5, -0.5, ny - 0.5), [-1.0, 0.0]),
        "east": (_rect(nx - 1.5, nx - 0.5, -0.5, ny - 0.5), [1.0, 0.0]),
        "south": (_rect(-0.5, nx - 0.5, -0.5, 0.5), [0.0, -1.0]),
        "north": (_rect(-0.5, nx - 0.5, ny - 1.5, ny - 0.5), [0.0, 1.0]),
    }
    out = {}
    for side, types in (("west", west), ("east", east), ("south", south), ("north", north)):
        poly, normal = polys[side]
        for t in types:
            if isinstance(t, tuple):
                t, vals = t
            else:
                vals = [0.0, 0.0, 0.0, 0.0]
            out[f"{side}_{t}"] = {"type": t, "polygon": poly, "values": list(vals), "normal": normal}
    return out


def index_coords(ny, nx):
    return np.meshgrid(np.arange(nx, dtype=np.float64), (ny - 1 - np.arange(ny)).astype(np.float64), indexing="xy")
