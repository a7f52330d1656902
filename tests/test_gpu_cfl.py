"""The two row-copy forms of the float32 CFL item give the same time step bit for bit
(GPU only).

States whose rows start on 16-byte boundaries (the default 32-element pitch) copy each row
of h, hu, hv and G into the warp's shared slots as 16-byte chunks, from lane 0's column
rounded down to a multiple of 4, and lanes read columns other lanes copied; any other
layout copies one element per lane and plane.  Both reduce the maximum of the same face
speeds (roe_exner.py:257-310 through compute_dt_2D) over the same faces, and a maximum
does not depend on the order it is taken in, so the dts must be equal.  The copy below
shifts every plane by one element (4 bytes) inside a wider allocation: same pitch, same
values, rows no longer 16-byte aligned.
"""
import numpy as np
import pytest
import torch

from helpers import random_re_case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _lib_built():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pyexner_b200 import build

    build.build()


def shifted(st):
    """The same state with every plane one element off the 16-byte row alignment."""
    kw = {}
    for f in st.PLANES:
        t = getattr(st, f)
        if t is None:
            kw[f] = None
            continue
        big = torch.zeros((t.shape[0], t.stride(0) + 4), dtype=t.dtype, device=t.device)
        view = torch.as_strided(big, t.shape, (t.stride(0), 1), storage_offset=1)
        view.copy_(t)
        kw[f] = view
    return st.replace(**kw)


def device_case(arrs, params, X, Y, dx=0.1):
    from pyexner_b200 import BoundaryManager, RoeExnerState, create_solver_bundle
    from pyexner_b200.cases import seds_matrix

    seds = seds_matrix(params["erosion"])
    bm = BoundaryManager(params, X, Y)
    st = RoeExnerState.from_numpy(arrs, seds, torch.float32)
    bundle = create_solver_bundle("Roe Exner")
    cfg = bundle.config(st, None, bm, dx, params)
    mask = bundle.mask_fn(st, None, bm.boundary_mask)
    return bundle, bundle.init_fn(st, mask, cfg), mask, cfg


def dt_bits(bundle, st, mask, cfg):
    return np.float32(float(bundle.compute_dt_fn(st, 0.5, mask, cfg))).view(np.uint32)


@pytest.mark.parametrize("shape,regime,bc,mpm", [
    ((70, 100), "fast", "trans_x_refl_y", True),
    ((131, 61), "wetdry", "refl_all", True),
    ((57, 83), "fast", "influx_left", False),
    ((64, 55), "wetdry", "partial_nodata", False),
    ((3, 3), "smooth", "refl_all", True),
    ((200, 3), "smooth", "trans_x_refl_y", True),
    ((3, 200), "smooth", "trans_x_refl_y", True),
    ((5, 257), "fast", "refl_all", True),
    ((129, 125), "fast", "trans_x_refl_y", False),
    ((300, 530), "wetdry", "trans_x_refl_y", True),
])
def test_chunked_rows_match_element_rows(shape, regime, bc, mpm):
    """Strip edges at every phase of the 16-byte chunks (31-column strips start at every
    column modulo 4), wet/dry cells, nodata cells, constant and MPM grass factors; the dt
    after each of 6 SSPRK2 steps too (bedload switching on in the fast cases)."""
    from pyexner_b200 import run_steps

    ny, nx = shape
    arrs, params, X, Y, mpm = random_re_case(ny, nx, seed=ny * 13 + nx, regime=regime, bcname=bc, mpm=mpm)
    bundle, st, mask, cfg = device_case(arrs, params, X, Y)
    for _ in range(7):
        sh = shifted(st)
        assert sh.h.data_ptr() % 16 != 0 and st.h.data_ptr() % 16 == 0
        assert dt_bits(bundle, st, mask, cfg) == dt_bits(bundle, sh, mask, cfg)
        run_steps(st, mask, cfg, "SSPRK2", 1, 0.5, log_dt=False)


@pytest.mark.parametrize("u0", [0.1, 0.55, 1.0])
def test_chunked_rows_gaussian_bed(u0):
    """The Gaussian-bed workload below, at and above the Shields threshold (the shallow-water
    speed, both forms side by side, the cubic everywhere)."""
    from pyexner_b200 import cases, run_steps

    c = cases.gaussian_bed(510, u0=u0)
    bundle, st, mask, cfg = device_case(c["arrs"], c["params"], c["X"], c["Y"], c["dx"])
    for _ in range(3):
        assert dt_bits(bundle, st, mask, cfg) == dt_bits(bundle, shifted(st), mask, cfg)
        run_steps(st, mask, cfg, "SSPRK2", 2, 0.5, log_dt=False)
