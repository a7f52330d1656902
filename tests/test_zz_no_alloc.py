"""The allocation-free time step, pxb_re_cfl_noalloc, against the plan-based pxb_re_cfl.

pxb_re_cfl_noalloc exists for callers that cannot allocate device memory when they ask
for dt: an XLA custom call working inside buffers XLA already owns, or an application
that forbids cudaMalloc after start-up.  It keeps its reduction scratch in a fixed device
array owned by the library, so two calls in a row must both reproduce the regular entry
point (the second call reuses the array the first one left behind), and the device's
free memory must not move across a call.  Both entry points evaluate the same faces with
the same arithmetic (float64 built with --fmad=false in both), and the maximum over faces
does not depend on the order of the reduction, so dt is compared bit for bit.  This file
is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest
import torch

from helpers import random_re_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32], ids=["f64", "f32"])
@pytest.mark.parametrize("shape,regime,bc", [((300, 251), "fast", "trans_x_refl_y"),
                                             ((90, 77), "wetdry", "partial_nodata")])
def test_noalloc_cfl_matches_plan_cfl_twice(dtype, shape, regime, bc):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from pyexner_b200 import BoundaryManager, RoeExnerState, _lib, build, create_solver_bundle
    from pyexner_b200.cases import seds_matrix

    build.build()
    ny, nx = shape
    arrs, params, X, Y, mpm = random_re_case(ny, nx, seed=ny + nx, regime=regime, bcname=bc)
    bm = BoundaryManager(params, X, Y)
    st = RoeExnerState.from_numpy(arrs, seds_matrix(params["erosion"]), dtype)
    bundle = create_solver_bundle("Roe Exner")
    cfg = bundle.config(st, None, bm, 0.1, params)
    mask = bundle.mask_fn(st, None, bm.boundary_mask)
    st = bundle.init_fn(st, mask, cfg)
    ref = float(bundle.compute_dt_fn(st, 0.5, mask, cfg))

    nodata = None
    if bool(mask[0].any()):
        from pyexner_b200.state import alloc_plane

        nodata = alloc_plane(ny, nx, torch.uint8, "cuda", align=st.pitch)  # same row pitch as the state
        nodata.copy_(mask[0].to(torch.uint8))
        assert nodata.stride(0) == st.pitch
    code = _lib.F64 if dtype == torch.float64 else _lib.F32
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    dt = torch.full((), -1.0, dtype=dtype, device="cuda")
    torch.cuda.synchronize()
    for call in range(2):
        dt.fill_(-1.0)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        _lib.call("pxb_re_cfl_noalloc", ny, nx, st.pitch, code, 0.1, 0.5, st.h.data_ptr(), st.hu.data_ptr(),
                  st.hv.data_ptr(), st.G.data_ptr(), nodata.data_ptr() if nodata is not None else None,
                  dt.data_ptr(), stream)
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info()[0]
        got = float(dt)
        assert got == ref, (call, got, ref)
        if call == 1:  # the first call may load the kernel's module; the second must not touch device memory
            assert free1 == free0, (free0, free1)
