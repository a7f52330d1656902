"""Host-side checks that need no GPU: the C ABI library, the boundary set-up, the cases."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from bc_specs import BC_SPECS, ROE_BC_SPECS, grid_coords
from oracle import boundaries as OB
from pyexner_b200 import _lib
from pyexner_b200.boundaries import BoundaryManager, roe_exner_mask


def test_library_exports_every_header_symbol():
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("library not built (python -m pyexner_b200.build)")
    names = _lib.header_symbols()
    assert "pxb_re_stage" in names and "pxb_re_run" in names
    lib = ctypes.CDLL(_lib.LIB_PATH)  # loading does not touch the GPU
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if " T " in l}
    assert set(names) <= exported
    assert set(_lib.SIGNATURES) | {"pxb_last_error"} == set(names)


def test_ctypes_structs_match_header_layout():
    assert ctypes.sizeof(_lib.BcHandler) == 120 and _lib.BcHandler.values.offset == 56
    assert ctypes.sizeof(_lib.REFields) == 64
    assert ctypes.sizeof(_lib.RoeFields) == 40
    assert _lib.REConfig.pitch.offset == 8 and _lib.REConfig.dx.offset == 24
    assert _lib.REConfig.handlers.offset == 56 and _lib.REConfig.stage_path.offset == 72
    assert ctypes.sizeof(_lib.REConfig) == 80


@pytest.mark.parametrize("name", sorted(BC_SPECS))
def test_boundary_setup_matches_oracle(name):
    ny, nx = 11, 14
    spec = BC_SPECS[name](ny, nx)
    X, Y = grid_coords(ny, nx)
    bm = BoundaryManager(dict(flux_scheme="Roe Exner", boundaries=spec), X, Y)
    ob = OB.Boundaries("Roe Exner", spec, X, Y)
    assert np.array_equal(bm.boundary_mask, ob.boundary_mask)
    for hd, oh in zip(bm.handlers, ob.handlers):
        assert hd["kind"] == oh.kind
        for a, b in zip(hd["cells"] + hd["donors"], oh.b + oh.i):
            assert np.array_equal(a, b)
    z = np.zeros((ny, nx))
    assert np.array_equal(roe_exner_mask(z, bm.boundary_mask), OB.roe_exner_mask(z.copy(), ob.boundary_mask))


def test_flat_indices_use_the_pitch():
    ny, nx = 9, 10
    X, Y = grid_coords(ny, nx)
    bm = BoundaryManager(dict(flux_scheme="Roe", boundaries=ROE_BC_SPECS["roe_refl_all"](ny, nx)), X, Y)
    arr, n = bm.c_array(pitch=32)
    assert n == 4
    cells = np.ctypeslib.as_array(ctypes.cast(arr[0].cells, ctypes.POINTER(ctypes.c_int64)), (arr[0].count,))
    by, bx = bm.handlers[0]["cells"]
    assert np.array_equal(cells, by * 32 + bx)


def test_gaussian_bed_case_is_seeded():
    from pyexner_b200 import cases

    a = cases.gaussian_bed_fields(62, seed_bed=3, seed_noise=4)
    b = cases.gaussian_bed_fields(62, seed_bed=3, seed_noise=4)
    for k in a:
        assert np.array_equal(a[k], b[k])
    assert a["h"].shape == (64, 64)
    assert np.all(a["z_b"] >= 0.05 - 1e-12)
    assert np.allclose(a["hu"], 0.1 * a["h"])


def test_noalloc_rejects_too_wide_grid_without_touching_the_gpu():
    """The allocation-free time step checks the grid against its fixed scratch first."""
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("library not built")
    lib = _lib.load()
    code = lib.pxb_re_cfl_noalloc(10, 300000, 300000, _lib.F32, 0.1, 0.5, None, None, None, None, None, None, None)
    assert code == _lib.ERR_ARG
    assert b"allocation-free limit" in lib.pxb_last_error()
