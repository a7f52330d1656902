"""ctypes binding of ``libpyexner_b200.so`` (the C ABI in include/pyexner_b200.h).

There is no fallback: if the library is missing or a CUDA device is absent the calls
raise.  The product path never computes on the CPU.
"""
from __future__ import annotations

import ctypes
import os
import re
from ctypes import POINTER, c_double, c_int, c_int32, c_int64, c_size_t, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpyexner_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "pyexner_b200.h")

OK, ERR_ARG, ERR_CUDA, ERR_NONFINITE, ERR_UNSUPPORTED = 0, 1, 2, 3, 4
F32, F64 = 0, 1
FE, SSPRK2 = 0, 1
PATH_AUTO, PATH_FUSED, PATH_GENERAL = 0, 1, 2
BC_KINDS = {
    "Roe Exner Reflective": 1,
    "Roe Exner Transmissive": 2,
    "Roe Exner TransmissiveBed": 3,
    "Roe Exner ConstantInflux": 4,
    "Roe Reflective": 5,
    "Roe Transmissive": 6,
    "Roe Exner ConstantOutflux": 7,
    "Roe Exner Berthon": 8,
    "Roe Exner NormalFlowDepth": 9,
    "Roe Exner SteepFall": 10,
    "Roe Exner ZeroMomentum": 11,
}


class BcHandler(ctypes.Structure):
    _fields_ = [
        ("kind", c_int32),
        ("count", c_int32),
        ("cells", c_void_p),
        ("donors", c_void_p),
        ("nx", c_double),
        ("ny", c_double),
        ("hu_const", c_double),
        ("hv_const", c_double),
        ("values", c_double * 8),
    ]


class ParamAdjoints(ctypes.Structure):
    _fields_ = [("seds_bar", c_void_p), ("values0_bar", c_void_p)]


class REFields(ctypes.Structure):
    _fields_ = [(n, c_void_p) for n in ("h", "hu", "hv", "z", "z_b", "n", "n_b", "G")]


class RoeFields(ctypes.Structure):
    _fields_ = [(n, c_void_p) for n in ("h", "hu", "hv", "z", "n")]


class REConfig(ctypes.Structure):
    _fields_ = [
        ("ny", c_int32),
        ("nx", c_int32),
        ("pitch", c_int64),
        ("dtype", c_int32),
        ("mpm", c_int32),
        ("dx", c_double),
        ("seds", c_void_p),
        ("nsed", c_int32),
        ("nodata", c_void_p),
        ("handlers", POINTER(BcHandler)),
        ("nhandlers", c_int32),
        ("band_rows", c_int32),
        ("stage_path", c_int32),
    ]


class RoeConfig(ctypes.Structure):
    _fields_ = [
        ("ny", c_int32),
        ("nx", c_int32),
        ("pitch", c_int64),
        ("dtype", c_int32),
        ("dx", c_double),
        ("handlers", POINTER(BcHandler)),
        ("nhandlers", c_int32),
    ]


class REMember(ctypes.Structure):
    _fields_ = [
        ("ny", c_int32),
        ("nx", c_int32),
        ("pitch", c_int64),
        ("dx", c_double),
        ("a", REFields),
        ("b", REFields),
        ("nodata", c_void_p),
        ("handlers", POINTER(BcHandler)),
        ("nhandlers", c_int32),
    ]


class REEnsConfig(ctypes.Structure):
    _fields_ = [
        ("dtype", c_int32),
        ("mpm", c_int32),
        ("seds", c_void_p),
        ("nsed", c_int32),
        ("members", POINTER(REMember)),
        ("nmembers", c_int32),
        ("band_rows", c_int32),
    ]


class TangentParams(ctypes.Structure):
    _fields_ = [("seds_dot", c_void_p), ("values0_dot", c_void_p)]


class PxbError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"pyexner_b200 error {code}: {msg}")
        self.code = code


_lib = None

# (name, argtypes) of every entry point declared in include/pyexner_b200.h
SIGNATURES = {
    "pxb_re_plan_create": [POINTER(REConfig), POINTER(c_void_p)],
    "pxb_re_plan_destroy": [c_void_p],
    "pxb_re_plan_workspace_size": [POINTER(REConfig), POINTER(c_size_t)],
    "pxb_re_plan_create_in": [POINTER(REConfig), c_void_p, c_size_t, POINTER(c_void_p)],
    "pxb_re_init": [c_void_p, POINTER(REFields), c_void_p],
    "pxb_re_plan_path": [c_void_p],
    "pxb_re_autotune": [c_void_p, POINTER(REFields), POINTER(REFields), c_void_p, POINTER(c_int32)],
    "pxb_re_cfl": [c_void_p, POINTER(REFields), c_double, c_void_p, c_void_p],
    "pxb_re_stage": [c_void_p, POINTER(REFields), POINTER(REFields), POINTER(REFields), c_void_p, c_double,
                     c_void_p],
    "pxb_re_run": [c_void_p, POINTER(REFields), POINTER(REFields), c_int32, c_int32, c_double, c_double, c_void_p,
                   c_void_p],
    "pxb_re_check": [c_void_p, c_void_p],
    "pxb_re_vjp_init": [c_void_p, POINTER(REFields), POINTER(REFields), c_void_p],
    "pxb_re_vjp_run": [c_void_p, POINTER(REFields), c_int32, c_int32, c_double, c_double, c_int32, POINTER(REFields),
                       c_void_p],
    "pxb_re_jvp_init": [c_void_p, POINTER(REFields), POINTER(REFields), c_void_p, c_void_p],
    "pxb_re_jvp_run": [c_void_p, POINTER(REFields), POINTER(REFields), c_int32, c_int32, c_double, c_double, c_void_p,
                       c_void_p, c_void_p, c_void_p],
    "pxb_roe_plan_create": [POINTER(RoeConfig), POINTER(c_void_p)],
    "pxb_roe_plan_destroy": [c_void_p],
    "pxb_roe_cfl": [c_void_p, POINTER(RoeFields), c_double, c_void_p, c_void_p],
    "pxb_roe_stage": [c_void_p, POINTER(RoeFields), POINTER(RoeFields), POINTER(RoeFields), c_void_p, c_void_p],
    "pxb_roe_run": [c_void_p, POINTER(RoeFields), POINTER(RoeFields), c_int32, c_int32, c_double, c_void_p, c_void_p],
    "pxb_roe_check": [c_void_p, c_void_p],
    "pxb_re_ens_create": [POINTER(REEnsConfig), POINTER(c_void_p)],
    "pxb_re_ens_destroy": [c_void_p],
    "pxb_re_ens_init": [c_void_p, c_void_p],
    "pxb_re_ens_autotune": [c_void_p, c_void_p, POINTER(c_int32)],
    "pxb_re_ens_run": [c_void_p, c_int32, c_int32, c_double, c_void_p, c_void_p],
    "pxb_re_ens_check": [c_void_p, c_void_p, POINTER(c_int32)],
    "pxb_re_cfl_noalloc": [c_int32, c_int32, c_int64, c_int32, c_double, c_double, c_void_p, c_void_p, c_void_p,
                           c_void_p, c_void_p, c_void_p, c_void_p],
    "pxb_label_polygons": [c_int32, c_int32, c_void_p, c_void_p, c_void_p, c_int32, c_int32, c_void_p, c_void_p,
                           c_int64, c_void_p],
    "pxb_version": [],
    "pxb_re_volume": [c_void_p, POINTER(REFields), POINTER(c_double), c_void_p],
    "pxb_re_vjp_run_params": [c_void_p, POINTER(REFields), c_int32, c_int32, c_double, c_double, c_int32,
                              POINTER(REFields), c_void_p, c_void_p],
    "pxb_re_vjp_init_params": [c_void_p, POINTER(REFields), POINTER(REFields), c_void_p, c_void_p],
    "pxb_re_set_budget": [c_void_p, c_void_p],
}


def header_symbols():
    """Names of the functions declared in include/pyexner_b200.h."""
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(pxb_\w+)\s*\(", txt, re.M)))


def load():
    """Load the library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m pyexner_b200.build` "
            "(the CUDA path is the only implementation)"
        )
    lib = ctypes.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = c_int
    lib.pxb_last_error.restype = ctypes.c_char_p
    lib.pxb_last_error.argtypes = []
    _lib = lib
    return lib


def check(code):
    if code != OK:
        msg = load().pxb_last_error().decode(errors="replace")
        raise PxbError(code, msg)


def call(name, *args):
    check(getattr(load(), name)(*args))
