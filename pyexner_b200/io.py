"""NetCDF3 state input / output, off the timed loop.

Follows src/PyExner/io/pnetcdf_reader.py on one rank: the mesh comes from the file's
``x`` / ``y`` coordinates (dh = round(x[1] - x[0], 5), cell centres x + dh/2 and
y - dh/2, :56-109); the state variables are read and cast to float32 as the reference
does (:166-169), ``G`` comes from ``erosion.grass_factor`` when absent (:126-131) and the
sediment matrix from the YAML (:136-162); frames are written per output time with nodata
cells set to NaN (:222-256).

Files are classic NetCDF3 (CDF-1 / 64-bit-offset CDF-2), which is what the reference's
case generators write (``to_netcdf(..., format="NETCDF3_64BIT")``).  Frames are copied
device -> pinned host memory on a side stream and written by a background thread, so the
solver does not wait for the file system.
"""
from __future__ import annotations

import threading
from dataclasses import dataclass

import numpy as np
import torch
from scipy.io import netcdf_file

from .cases import seds_matrix

STATE_VARS = ("h", "hu", "hv", "z", "z_b", "n", "n_b", "G")


@dataclass
class Mesh2D:
    """src/PyExner/domain/mesh.py:10-24 (single rank: local = global)."""

    global_Ny: int
    global_Nx: int
    local_Ny: int
    local_Nx: int
    x_offset: int
    y_offset: int
    local_X: np.ndarray
    local_Y: np.ndarray
    dh: float
    local_shape: tuple
    global_shape: tuple


class NetCDFStateIO:
    def __init__(self, in_file_path, out_file_path=None):
        self.in_file_path = in_file_path
        self.out_file_path = out_file_path
        self.numOut = 0
        self._out = None
        self._vars = {}
        self._lock = threading.Lock()
        self._thread = None
        self._stream = None
        self._pinned = {}

    # ------------------------------------------------------------------ input
    def generate_mesh(self):
        with netcdf_file(self.in_file_path, "r", mmap=False) as f:
            x = np.array(f.variables["x"][:], dtype=np.float64)
            y = np.array(f.variables["y"][:], dtype=np.float64)
        dh = round(float((x[1:] - x[:-1])[0]), 5)
        X, Y = np.meshgrid(x + dh / 2, y - dh / 2, indexing="xy")
        ny, nx = len(y), len(x)
        self._x, self._y = x, y
        return Mesh2D(ny, nx, ny, nx, 0, 0, X, Y, dh, (ny, nx), (ny, nx))

    def read_state(self, state_cls, mesh, params, dtype=torch.float32, device="cuda"):
        erosion = params.get("erosion", {"grass_factor": 0.0})
        arrs = {}
        with netcdf_file(self.in_file_path, "r", mmap=False) as f:
            for name in ("h", "hu", "hv", "z", "z_b", "n", "G"):
                if name in f.variables:
                    arrs[name] = np.array(f.variables[name][:], dtype=np.float32).astype(np.float64)
        shape = mesh.local_shape
        for name in ("h", "hu", "hv", "z", "n"):
            if name not in arrs:
                raise KeyError(f"Variable '{name}' not found in NetCDF file.")
        if "z_b" not in arrs:
            arrs["z_b"] = np.zeros(shape)
        if "G" not in arrs:
            g = erosion.get("grass_factor", 0.0)
            arrs["G"] = np.zeros(shape) if isinstance(g, str) else float(g) * np.ones(shape)
        return state_cls.from_numpy(arrs, seds_matrix(erosion), dtype, device)

    # ------------------------------------------------------------------ output
    def _open_out(self, mesh, dtype):
        self._out = netcdf_file(self.out_file_path, "w", version=2)
        self._out.createDimension("t", None)
        self._out.createDimension("y", mesh.global_Ny)
        self._out.createDimension("x", mesh.global_Nx)
        vy = self._out.createVariable("y", "d", ("y",))
        vx = self._out.createVariable("x", "d", ("x",))
        vy[:] = self._y
        vx[:] = self._x
        for name in self._planes:
            self._vars[name] = self._out.createVariable(name, "f", ("t", "y", "x"))

    def write_state(self, state, mesh, mask):
        """Queue one output frame (nodata cells as NaN); returns without waiting for disk."""
        if self.out_file_path is None:
            return
        if self._out is None:
            self._planes = tuple(state.PLANES)
            self._open_out(mesh, state.dtype)
            self._stream = torch.cuda.Stream()
        m = mask.to(torch.bool) if isinstance(mask, torch.Tensor) else torch.as_tensor(mask, device=state.h.device)
        ev = torch.cuda.Event()
        ev.record()
        frames = {}
        with torch.cuda.stream(self._stream):
            self._stream.wait_event(ev)
            for name in self._planes:
                src = getattr(state, name)
                buf = torch.empty(src.shape, dtype=torch.float32, pin_memory=True)
                buf.copy_(torch.where(m, torch.nan, src).to(torch.float32), non_blocking=True)
                frames[name] = buf
            done = torch.cuda.Event()
            done.record(self._stream)
        k = self.numOut
        self.numOut += 1
        self.flush()

        def write():
            done.synchronize()
            with self._lock:
                for name, buf in frames.items():
                    self._vars[name][k] = buf.numpy()
                self._out.flush()

        self._thread = threading.Thread(target=write, daemon=True)
        self._thread.start()

    def flush(self):
        if self._thread is not None:
            self._thread.join()
            self._thread = None

    def close(self):
        self.flush()
        if self._out is not None:
            self._out.close()
            self._out = None


def write_input(path, x, y, fields):
    """Write a NETCDF3_64BIT input file in the reference's layout (float32 planes on
    (y, x) plus float32 ``x`` / ``y`` coordinates)."""
    with netcdf_file(path, "w", version=2) as f:
        f.createDimension("y", len(y))
        f.createDimension("x", len(x))
        vx = f.createVariable("x", "f", ("x",))
        vy = f.createVariable("y", "f", ("y",))
        vx[:] = np.asarray(x, dtype=np.float32)
        vy[:] = np.asarray(y, dtype=np.float32)
        for name, arr in fields.items():
            v = f.createVariable(name, "f", ("y", "x"))
            v[:] = np.asarray(arr, dtype=np.float32)
