"""State containers (device planes) mirroring PyExner's pytrees.

``RoeExnerState`` follows src/PyExner/state/roe_exner_state.py:8-48 (leaves h, hu, hv,
z, z_b, n, n_b, G, seds) and ``RoeState`` src/PyExner/state/roe_state.py:8-61 (h, hu,
hv, z, n).  Planes are torch CUDA tensors of shape (ny, nx), ring included, whose rows
may be padded to a pitch of 32 elements (128 B in float32) for aligned rows; the pitch
is the tensor's row stride.  ``seds`` stays a host float64 matrix (7 x nsed).
"""
from __future__ import annotations

import dataclasses
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib

STATE_REGISTRY = {}


def register_state(name):
    def deco(cls):
        STATE_REGISTRY[name] = cls
        return cls

    return deco


def create_state(name, params):
    return STATE_REGISTRY[name].from_params(params)


def torch_dtype(dtype):
    if dtype in (torch.float32, "float32", "fp32", np.float32):
        return torch.float32
    if dtype in (torch.float64, "float64", "fp64", np.float64):
        return torch.float64
    raise ValueError(f"unsupported dtype {dtype}")


def alloc_plane(ny, nx, dtype, device="cuda", align=32):
    pitch = ((nx + align - 1) // align) * align
    return torch.zeros((ny, pitch), dtype=dtype, device=device)[:, :nx]


def plane_from(arr, dtype, device="cuda"):
    arr = np.asarray(arr)
    t = alloc_plane(arr.shape[0], arr.shape[1], dtype, device)
    t.copy_(torch.from_numpy(np.ascontiguousarray(arr)).to(dtype))
    return t


class _Planes:
    PLANES: tuple = ()

    def replace(self, **kw):
        return dataclasses.replace(self, **kw)

    @property
    def shape(self):
        return tuple(self.h.shape)

    @property
    def pitch(self):
        return self.h.stride(0)

    @property
    def dtype(self):
        return self.h.dtype

    def check_layout(self):
        for f in self.PLANES:
            t = getattr(self, f)
            if t is None:
                continue
            if not t.is_cuda:
                raise ValueError(f"{f} is not a CUDA tensor")
            if t.dtype != self.h.dtype or tuple(t.shape) != self.shape or t.stride() != (self.pitch, 1):
                raise ValueError(f"{f} does not share dtype/shape/pitch with h")

    def to_numpy(self):
        out = {f: getattr(self, f).detach().cpu().numpy().astype(np.float64) for f in self.PLANES}
        return out

    def clone(self):
        kw = {}
        for fld in dataclasses.fields(self):
            v = getattr(self, fld.name)
            if isinstance(v, torch.Tensor):
                c = alloc_plane(v.shape[0], v.shape[1], v.dtype, v.device)
                c.copy_(v)
                v = c
            kw[fld.name] = v
        return type(self)(**kw)


@register_state("Roe Exner")
@dataclass
class RoeExnerState(_Planes):
    h: torch.Tensor
    hu: torch.Tensor
    hv: torch.Tensor
    z: torch.Tensor
    z_b: torch.Tensor
    n: torch.Tensor
    n_b: torch.Tensor
    G: torch.Tensor
    seds: np.ndarray

    PLANES = ("h", "hu", "hv", "z", "z_b", "n", "n_b", "G")

    @classmethod
    def from_numpy(cls, arrs, seds, dtype=torch.float32, device="cuda"):
        dtype = torch_dtype(dtype)
        ny, nx = np.shape(arrs["h"])
        kw = {}
        for f in cls.PLANES:
            a = arrs.get(f)
            kw[f] = plane_from(a if a is not None else np.zeros((ny, nx)), dtype, device)
        return cls(**kw, seds=np.asarray(seds, dtype=np.float64))

    @classmethod
    def empty(cls, shape, dtype=torch.float32, device="cuda", seds=None):
        """Flat-bed default (roe_exner_state.py:19-34): zeros, z = 1."""
        dtype = torch_dtype(dtype)
        kw = {f: alloc_plane(shape[0], shape[1], dtype, device) for f in cls.PLANES}
        kw["z"].fill_(1.0)
        return cls(**kw, seds=np.zeros((1, 1)) if seds is None else seds)

    def c_fields(self):
        return _lib.REFields(*[getattr(self, f).data_ptr() if getattr(self, f) is not None else None
                               for f in self.PLANES])


@register_state("Roe")
@dataclass
class RoeState(_Planes):
    h: torch.Tensor
    hu: torch.Tensor
    hv: torch.Tensor
    z: torch.Tensor
    n: torch.Tensor

    PLANES = ("h", "hu", "hv", "z", "n")

    @classmethod
    def from_numpy(cls, arrs, dtype=torch.float64, device="cuda"):
        dtype = torch_dtype(dtype)
        return cls(**{f: plane_from(arrs[f], dtype, device) for f in cls.PLANES})

    @classmethod
    def empty(cls, shape, dtype=torch.float64, device="cuda"):
        dtype = torch_dtype(dtype)
        kw = {f: alloc_plane(shape[0], shape[1], dtype, device) for f in cls.PLANES}
        kw["z"].fill_(1.0)
        return cls(**kw)

    def c_fields(self):
        return _lib.RoeFields(*[getattr(self, f).data_ptr() for f in self.PLANES])
