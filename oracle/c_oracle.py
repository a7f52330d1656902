"""ctypes wrapper of the C / OpenMP oracle (oracle/c/re_oracle.c); test infrastructure.

``build()`` compiles it with gcc (-O2 -fopenmp -ffp-contract=off) into oracle/c/build/.
``run_roe_exner`` mirrors ``oracle.integrators.run_roe_exner`` and is used as the
multi-threaded CPU baseline of bench.py.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "c", "re_oracle.c")
OUT = os.path.join(HERE, "c", "build", "libre_oracle.so")

KINDS = {"Roe Exner Reflective": 1, "Roe Exner Transmissive": 2, "Roe Exner TransmissiveBed": 3,
         "Roe Exner ConstantInflux": 4}


class _Handler(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("count", ctypes.c_int32), ("cells", ctypes.c_void_p),
                ("donors", ctypes.c_void_p), ("nx", ctypes.c_double), ("ny", ctypes.c_double),
                ("hu_const", ctypes.c_double), ("hv_const", ctypes.c_double)]


class _Case(ctypes.Structure):
    _fields_ = [("ny", ctypes.c_int), ("nx", ctypes.c_int), ("mpm", ctypes.c_int), ("nsed", ctypes.c_int),
                ("dx", ctypes.c_double), ("seds", ctypes.c_void_p), ("nodata", ctypes.c_void_p),
                ("hs", ctypes.POINTER(_Handler)), ("nh", ctypes.c_int)]


class _State(ctypes.Structure):
    _fields_ = [(n, ctypes.c_void_p) for n in ("h", "hu", "hv", "z", "zb", "n", "nb", "G")]


OUT32 = os.path.join(HERE, "c", "build", "libre_oracle_f32.so")


def build(force=False):
    """Both builds of the restatement: float64 (the oracle) and float32 (the same
    operations on a float32 state, as the reference runs as shipped)."""
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    for out, real in ((OUT, "double"), (OUT32, "float")):
        if not force and os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(SRC):
            continue
        subprocess.run(["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
                        f"-DOC_REAL={real}", SRC, "-o", out, "-lm"], check=True)
    return OUT


_libs = {}


def lib(dtype=np.float64):
    key = np.dtype(dtype).name
    if key not in _libs:
        build()
        L = ctypes.CDLL(OUT if key == "float64" else OUT32)
        L.oc_re_run.argtypes = [ctypes.POINTER(_Case), ctypes.POINTER(_State), ctypes.c_int, ctypes.c_int,
                                ctypes.c_double, ctypes.c_void_p]
        L.oc_re_run.restype = ctypes.c_int
        L.oc_re_init.argtypes = [ctypes.POINTER(_Case), ctypes.POINTER(_State)]
        _libs[key] = L
    return _libs[key]


def _case(shape, bcs, mask0, mpm, seds, dx, keep):
    ny, nx = shape
    hs = (_Handler * max(1, len(bcs.handlers)))()
    for k, hd in enumerate(bcs.handlers):
        by, bx = hd.b
        iy, ix = hd.i
        cells = np.ascontiguousarray(by.astype(np.int64) * nx + bx)
        donors = np.ascontiguousarray(iy.astype(np.int64) * nx + ix)
        keep += [cells, donors]
        hs[k].kind = KINDS[hd.kind]
        hs[k].count = len(cells)
        hs[k].cells = cells.ctypes.data
        hs[k].donors = donors.ctypes.data
        hs[k].nx, hs[k].ny = float(hd.normal[0]), float(hd.normal[1])
        if hd.kind == "Roe Exner ConstantInflux":
            hs[k].hu_const = float(np.float32(hd.values[0]) * np.float32(hd.values[1]))
            hs[k].hv_const = float(np.float32(hd.values[0]) * np.float32(hd.values[2]))
    keep.append(hs)
    sd = np.ascontiguousarray(np.asarray(seds, dtype=np.float64))
    keep.append(sd)
    nod = None
    if mask0 is not None and mask0.any():
        nod = np.ascontiguousarray(mask0.astype(np.uint8))
        keep.append(nod)
    c = _Case(ny, nx, 1 if mpm else 0, sd.shape[1] if mpm else 0, dx, sd.ctypes.data if mpm else None,
              nod.ctypes.data if nod is not None else None, hs, len(bcs.handlers))
    return c


def _state(st, keep, dtype=np.float64):
    arrs = {k: np.ascontiguousarray(np.array(st[k], dtype=dtype)) for k in
            ("h", "hu", "hv", "z", "z_b", "n", "n_b", "G")}
    keep.append(arrs)
    s = _State(*[arrs[k].ctypes.data for k in ("h", "hu", "hv", "z", "z_b", "n", "n_b", "G")])
    return s, arrs


def init(st, mask, bcs, mpm, dx=1.0, dtype=np.float64):
    keep = []
    c = _case(st["h"].shape, bcs, mask[0], mpm, st["seds"], dx, keep)
    s, arrs = _state(st, keep, dtype)
    lib(dtype).oc_re_init(ctypes.byref(c), ctypes.byref(s))
    out = dict(arrs)
    out["seds"] = st["seds"]
    return out


def run_roe_exner(st, mask, bcs, mpm, dx, cfl, nsteps, scheme, dtype=np.float64):
    """Same contract as oracle.integrators.run_roe_exner (st must already be initialised);
    dtype np.float32 runs the float32 build on a float32 copy of the state."""
    keep = []
    c = _case(st["h"].shape, bcs, mask[0], mpm, st["seds"], dx, keep)
    s, arrs = _state(st, keep, dtype)
    dts = np.zeros(max(1, nsteps))
    rc = lib(dtype).oc_re_run(ctypes.byref(c), ctypes.byref(s), int(nsteps), 1 if scheme == "SSPRK2" else 0, float(cfl),
                         dts.ctypes.data)
    if rc != 0:
        raise MemoryError("C oracle: allocation failed")
    out = dict(arrs)
    out["seds"] = st["seds"]
    return out, dts[:nsteps]
