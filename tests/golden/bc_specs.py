"""Boundary layouts for the golden cases, written as PyExner YAML ``boundaries`` dicts.

Cell centres sit at integer coordinates: ``X = column``, ``Y = (ny - 1 - row)``, so
row 0 is the top (largest y) and the y-face normal (0, -1) points from row r to
row r + 1, as in src/PyExner/solvers/kernels/roe_exner.py:577.  Polygon edges sit on
half-integers so no cell centre is on an edge.  Normals are outward.
"""
import numpy as np


def grid_coords(ny, nx):
    X, Y = np.meshgrid(np.arange(nx, dtype=np.float64), (ny - 1 - np.arange(ny)).astype(np.float64), indexing="xy")
    return X, Y


def _rect(x0, x1, y0, y1):
    return [[x0, y0], [x1, y0], [x1, y1], [x0, y1]]


def left(ny, nx, rows=None):
    y0, y1 = (-0.5, ny - 0.5) if rows is None else (ny - 1 - rows[1] - 0.5, ny - 1 - rows[0] + 0.5)
    return _rect(-0.5, 0.5, y0, y1)


def right(ny, nx, rows=None):
    y0, y1 = (-0.5, ny - 0.5) if rows is None else (ny - 1 - rows[1] - 0.5, ny - 1 - rows[0] + 0.5)
    return _rect(nx - 1.5, nx - 0.5, y0, y1)


def top(ny, nx, cols=None):
    x0, x1 = (-0.5, nx - 0.5) if cols is None else (cols[0] - 0.5, cols[1] + 0.5)
    return _rect(x0, x1, ny - 1.5, ny - 0.5)


def bottom(ny, nx, cols=None):
    x0, x1 = (-0.5, nx - 0.5) if cols is None else (cols[0] - 0.5, cols[1] + 0.5)
    return _rect(x0, x1, -0.5, 0.5)


def _b(t, poly, normal, values=(0.0, 0.0, 0.0, 0.0)):
    return {"type": t, "polygon": poly, "values": list(values), "normal": list(normal)}


def trans_x_refl_y(ny, nx):
    """Transmissive + TransmissiveBed in x, Reflective in y applied last (wins corners)."""
    return {
        "west": _b("Transmissive", left(ny, nx), [-1.0, 0.0]),
        "west_bed": _b("TransmissiveBed", left(ny, nx), [-1.0, 0.0]),
        "east": _b("Transmissive", right(ny, nx), [1.0, 0.0]),
        "east_bed": _b("TransmissiveBed", right(ny, nx), [1.0, 0.0]),
        "south": _b("Reflective", bottom(ny, nx), [0.0, -1.0]),
        "north": _b("Reflective", top(ny, nx), [0.0, 1.0]),
    }


def refl_first(ny, nx):
    """Reflective walls first, transmissive sides afterwards (the other corner order)."""
    return {
        "north": _b("Reflective", top(ny, nx), [0.0, 1.0]),
        "south": _b("Reflective", bottom(ny, nx), [0.0, -1.0]),
        "west": _b("Transmissive", left(ny, nx), [-1.0, 0.0]),
        "east_bed": _b("TransmissiveBed", right(ny, nx), [1.0, 0.0]),
        "east": _b("Transmissive", right(ny, nx), [1.0, 0.0]),
        "west_bed": _b("TransmissiveBed", left(ny, nx), [-1.0, 0.0]),
    }


def refl_all(ny, nx):
    return {
        "outlet1": _b("Reflective", left(ny, nx), [-1.0, 0.0]),
        "outlet2": _b("Reflective", right(ny, nx), [1.0, 0.0]),
        "outlet3": _b("Reflective", bottom(ny, nx), [0.0, -1.0]),
        "outlet4": _b("Reflective", top(ny, nx), [0.0, 1.0]),
    }


def influx_left(ny, nx):
    return {
        "inlet": _b("ConstantInflux", left(ny, nx), [-1.0, 0.0], values=(0.35, 1.0, 0.0)),
        "inlet_bed": _b("TransmissiveBed", left(ny, nx), [-1.0, 0.0]),
        "outlet": _b("Transmissive", right(ny, nx), [1.0, 0.0]),
        "outlet_bed": _b("TransmissiveBed", right(ny, nx), [1.0, 0.0]),
        "south": _b("Reflective", bottom(ny, nx), [0.0, -1.0]),
        "north": _b("Reflective", top(ny, nx), [0.0, 1.0]),
    }


def partial_nodata(ny, nx):
    """Walls that stop one cell short of the corners: the four corners become nodata."""
    return {
        "south": _b("Reflective", bottom(ny, nx, cols=(1, nx - 2)), [0.0, -1.0]),
        "north": _b("Reflective", top(ny, nx, cols=(1, nx - 2)), [0.0, 1.0]),
        "west": _b("Transmissive", left(ny, nx, rows=(1, ny - 2)), [-1.0, 0.0]),
        "west_bed": _b("TransmissiveBed", left(ny, nx, rows=(1, ny - 2)), [-1.0, 0.0]),
        "east": _b("Reflective", right(ny, nx, rows=(1, ny - 2)), [1.0, 0.0]),
    }


def refl_self(ny, nx):
    """Reflective walls whose y-normals point into the grid, as in the reference's
    dam-break inputs (ascending y in the file): the donor clips to the cell itself."""
    return {
        "outlet1": _b("Reflective", left(ny, nx), [-1.0, 0.0]),
        "outlet2": _b("Reflective", right(ny, nx), [1.0, 0.0]),
        "outlet3": _b("Reflective", top(ny, nx), [0.0, -1.0]),
        "outlet4": _b("Reflective", bottom(ny, nx), [0.0, 1.0]),
    }


def berthon_like(ny, nx):
    """The inlet / outlet layout of the reference's Berthon analytic case
    (tests/runtime/2D_const_flux/input.yaml): ConstantInflux + Berthon bed on the left,
    NormalFlowDepth on the right, reflective walls."""
    return {
        "inlet_flux": _b("ConstantInflux", left(ny, nx), [-1.0, 0.0], values=(1.0, 1.0, 0.0)),
        "inlet_bed": _b("Berthon", left(ny, nx), [-1.0, 0.0], values=(1.0, 0.005, 0.005, 0.005, 1, 0.0)),
        "outlet_bed": _b("NormalFlowDepth", right(ny, nx), [1.0, 0.0],
                         values=(1.0, 0.005, 0.005, 0.005, 1, float(nx - 1))),
        "bottom": _b("Reflective", bottom(ny, nx), [0.0, -1.0]),
        "top": _b("Reflective", top(ny, nx), [0.0, 1.0]),
    }


def outflux_steep(ny, nx):
    """ConstantOutflux + SteepFall outlet, zero-momentum walls (one with NaN values,
    which leaves the momentum as it is)."""
    return {
        "inlet": _b("ConstantInflux", left(ny, nx), [-1.0, 0.0], values=(0.3, 1.0, 0.0)),
        "inlet_bed": _b("TransmissiveBed", left(ny, nx), [-1.0, 0.0]),
        "outlet": _b("ConstantOutflux", right(ny, nx), [1.0, 0.0], values=(0.3, 1.0, 0.0)),
        "fall": _b("SteepFall", right(ny, nx), [1.0, 0.0]),
        "top": _b("ZeroMomentum", top(ny, nx), [0.0, 1.0], values=(0.0, 0.0, 0.0, 0.0)),
        "bottom_keep": _b("ZeroMomentum", bottom(ny, nx), [0.0, -1.0],
                          values=("nan", "nan", "nan", "nan")),
        "bottom": _b("Reflective", bottom(ny, nx), [0.0, -1.0]),
    }


def l_domain(ny, nx):
    """An L-shaped domain: the top-right block (rows 0-5, columns >= nx-6) has a NaN bed
    (nodata); walls follow the L, including an interior wall along the block's left side
    and an interior floor under it, as in the reference's L-domain cases."""
    bx0 = nx - 6  # first nodata column
    return {
        "left": _b("Reflective", left(ny, nx), [-1.0, 0.0]),
        "bottom": _b("Reflective", bottom(ny, nx), [0.0, -1.0]),
        "top": _b("Reflective", top(ny, nx, cols=(0, bx0 - 1)), [0.0, 1.0]),
        "right": _b("Reflective", right(ny, nx, rows=(6, ny - 1)), [1.0, 0.0]),
        "internal_wall": _b("Reflective", [[bx0 - 1.5, ny - 6.5], [bx0 - 0.5, ny - 6.5], [bx0 - 0.5, ny - 1.5],
                                            [bx0 - 1.5, ny - 1.5]], [1.0, 0.0]),
        "internal_floor": _b("Reflective", [[bx0 - 0.5, ny - 7.5], [nx - 1.5, ny - 7.5], [nx - 1.5, ny - 6.5],
                                             [bx0 - 0.5, ny - 6.5]], [0.0, 1.0]),
    }


BC_SPECS = {
    "berthon_like": berthon_like,
    "outflux_steep": outflux_steep,
    "l_domain": l_domain,
    "refl_self": refl_self,
    "trans_x_refl_y": trans_x_refl_y,
    "refl_first": refl_first,
    "refl_all": refl_all,
    "influx_left": influx_left,
    "partial_nodata": partial_nodata,
}


def roe_refl_all(ny, nx):
    return {
        "left": _b("Reflective", left(ny, nx), [-1.0, 0.0]),
        "right": _b("Reflective", right(ny, nx), [1.0, 0.0]),
        "bottom": _b("Reflective", bottom(ny, nx), [0.0, -1.0]),
        "top": _b("Reflective", top(ny, nx), [0.0, 1.0]),
    }


def roe_trans_x_refl_y(ny, nx):
    return {
        "west": _b("Transmissive", left(ny, nx), [-1.0, 0.0]),
        "east": _b("Transmissive", right(ny, nx), [1.0, 0.0]),
        "south": _b("Reflective", bottom(ny, nx), [0.0, -1.0]),
        "north": _b("Reflective", top(ny, nx), [0.0, 1.0]),
    }


ROE_BC_SPECS = {"roe_refl_all": roe_refl_all, "roe_trans_x_refl_y": roe_trans_x_refl_y}
