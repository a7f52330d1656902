"""Ragged ensembles of Roe-Exner grids on one GPU (``pxb_re_ens_*`` of the C ABI).

The reference runs one grid per process; an ensemble here is many independent grids
(their own sizes, states, boundary handlers and dts) advanced together, one launch per
phase (CFL, stage 1, stage 2) for all of them, the steps captured in a CUDA graph.  Each
member gives the same numbers as a run of its own through ``run_steps``.

    ens = Ensemble(members, erosion, dtype=torch.float32)
    ens.init()                 # init_fn_roeexner of every member
    ens.autotune()             # band height of the stage kernel, timed on the GPU
    dts = ens.run(1000, "SSPRK2", cfl=0.5)   # (steps, members) device tensor of dts
    ens.check()

``members``: a list of dicts with ``state`` (RoeExnerState on the device), ``boundaries``
(BoundaryManager of its YAML ``boundaries`` block) and ``dx``.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .boundaries import roe_exner_mask
from .integrators import scratch_like
from .solvers import _dtype_code, _stream
from .state import alloc_plane


def partition_members(cells, world):
    """Split ensemble members over ``world`` ranks (one process per GPU, replicas only:
    no data crosses ranks).  ``cells``: the cell count of every member.  Returns one
    sorted list of member indices per rank: members are dealt largest first to the rank
    with the fewest cells so far (ties to the lower rank), so every rank computes the same
    split on its own and the ranks finish close together."""
    if world < 1:
        raise ValueError("world must be at least 1")
    load = [0] * world
    parts = [[] for _ in range(world)]
    for k in sorted(range(len(cells)), key=lambda i: (-int(cells[i]), i)):
        r = min(range(world), key=lambda j: (load[j], j))
        parts[r].append(k)
        load[r] += int(cells[k])
    return [sorted(p) for p in parts]


class Ensemble:
    def __init__(self, members, erosion, dtype=None, band_rows=0):
        if not members:
            raise ValueError("an ensemble needs at least one member")
        self.members = members
        st0 = members[0]["state"]
        self.dtype = dtype if dtype is not None else st0.dtype
        grass = erosion.get("grass_factor", 0.0)
        self.mpm = isinstance(grass, str)
        self.seds = np.ascontiguousarray(np.asarray(st0.seds, dtype=np.float64))
        self.scratch = []
        self._keep = []
        arr = (_lib.REMember * len(members))()
        for k, mb in enumerate(members):
            st = mb["state"]
            if st.dtype != self.dtype:
                raise ValueError(f"member {k}: dtype {st.dtype} differs from the ensemble's {self.dtype}")
            st.check_layout()
            ny, nx = st.shape
            b = scratch_like(st)
            self.scratch.append(b)
            bm = mb["boundaries"]
            handlers, nh = bm.c_array(st.pitch) if bm is not None else (None, 0)
            z = st.z.detach().cpu().numpy()
            m0 = roe_exner_mask(z, bm.boundary_mask if bm is not None else np.zeros(z.shape, bool))[0]
            nod = None
            if m0.any():
                nod = alloc_plane(ny, nx, torch.uint8, st.h.device, align=st.pitch)
                nod.copy_(torch.from_numpy(m0.astype(np.uint8)))
            self._keep += [handlers, nod]
            arr[k].ny, arr[k].nx, arr[k].pitch = ny, nx, st.pitch
            arr[k].dx = float(mb["dx"])
            arr[k].a = st.c_fields()
            arr[k].b = b.c_fields()
            arr[k].nodata = nod.data_ptr() if nod is not None else None
            arr[k].handlers = handlers if nh else None
            arr[k].nhandlers = nh
        self._members_c = arr
        cfg = _lib.REEnsConfig()
        cfg.dtype = _dtype_code(self.dtype)
        cfg.mpm = 1 if self.mpm else 0
        cfg.seds = self.seds.ctypes.data_as(ctypes.c_void_p) if self.mpm else None
        cfg.nsed = self.seds.shape[1] if self.mpm else 0
        cfg.members = arr
        cfg.nmembers = len(members)
        cfg.band_rows = int(band_rows)
        h = ctypes.c_void_p()
        _lib.call("pxb_re_ens_create", ctypes.byref(cfg), ctypes.byref(h))
        self.handle = h
        self.band_rows = int(band_rows) if band_rows else None

    def __len__(self):
        return len(self.members)

    def __del__(self):
        try:
            if getattr(self, "handle", None) is not None and self.handle.value:
                _lib.load().pxb_re_ens_destroy(self.handle)
        except Exception:
            pass

    def init(self):
        _lib.call("pxb_re_ens_init", self.handle, _stream())

    def autotune(self):
        out = ctypes.c_int32(0)
        _lib.call("pxb_re_ens_autotune", self.handle, _stream(), ctypes.byref(out))
        self.band_rows = int(out.value)
        return self.band_rows

    def run(self, n_steps, scheme="SSPRK2", cfl=0.5, log_dt=True):
        code = _lib.SSPRK2 if scheme == "SSPRK2" else _lib.FE
        dev = self.members[0]["state"].h.device
        dts = torch.empty((max(1, n_steps), len(self)), dtype=self.dtype, device=dev) if log_dt else None
        _lib.call("pxb_re_ens_run", self.handle, int(n_steps), code, float(cfl),
                  ctypes.c_void_p(dts.data_ptr()) if dts is not None else None, _stream())
        return dts[:n_steps] if dts is not None else None

    def check(self):
        bad = ctypes.c_int32(-1)
        _lib.call("pxb_re_ens_check", self.handle, _stream(), ctypes.byref(bad))

    def cells(self):
        """Physical cells of all members (ring excluded)."""
        return sum((m["state"].shape[0] - 2) * (m["state"].shape[1] - 2) for m in self.members)
