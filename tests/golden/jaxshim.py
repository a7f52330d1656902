"""A small numpy-backed stand-in for the parts of JAX that PyExner's kernels use.

Purpose: JAX is not installed in this container, but PyExner (the reference) is pure
Python on ``jax.numpy``.  Installing this shim in ``sys.modules`` lets the reference's
own modules (``solvers/kernels/roe_exner.py``, ``solvers/kernels/roe.py``,
``solvers/roe_exner_solver.py``, ``solvers/roe_solver.py``, the boundary handlers)
be imported and executed on float64 numpy arrays, which is what
``jax.config.update("jax_enable_x64", True)`` gives on CPU up to XLA's own rounding.

It is used only by ``tests/golden/make_golden.py`` to generate the golden vectors
that pin the oracle.  Nothing in the product imports it.

Semantics kept from JAX:
  * ``x ** k`` with a Python int ``k`` is ``lax.integer_pow`` (repeated multiplication);
    other exponents go to ``pow``.
  * ``x.at[idx].set(v)`` / ``.add(v)`` are functional (return a new array);
    ``.add`` accumulates duplicates like ``jax.numpy`` scatter-add.
  * ``jit`` / ``vmap`` / ``lax.fori_loop`` / ``lax.while_loop`` have their
    mathematical meaning (no tracing).
  * MPI entry points used on one rank (``allreduce``, ``sendrecv``) are identities.
"""
from __future__ import annotations

import functools
import sys
import types

import numpy as np


class JArr(np.ndarray):
    """ndarray with the functional ``.at[...]`` update syntax of jax arrays."""

    @property
    def at(self):
        return _At(self)

    def __pow__(self, y):
        # ``x ** k`` with a Python int k is ``lax.integer_pow`` in JAX: powering by
        # repeated multiplication, not a call of pow().
        if isinstance(y, int) and not isinstance(y, bool):
            return _integer_pow(self, y)
        return _wrap(np.power(self, y))


def _integer_pow(x, y):
    """jax.lax.integer_pow: binary powering (x**3 = x * (x * x)), reciprocal for y < 0."""
    if y == 0:
        return _wrap(np.ones_like(x))
    recip = y < 0
    y = -y if recip else y
    acc = None
    while y > 0:
        if y & 1:
            acc = x if acc is None else np.multiply(acc, x)
        y >>= 1
        if y > 0:
            x = np.multiply(x, x)
    return _wrap(np.divide(np.ones_like(acc), acc) if recip else acc)


class _At:
    def __init__(self, arr):
        self._arr = arr

    def __getitem__(self, idx):
        return _AtIdx(self._arr, idx)


def _norm_idx(idx):
    # jnp accepts tuples of index arrays (from argwhere columns); numpy too.
    if isinstance(idx, tuple):
        return tuple(np.asarray(i) if isinstance(i, (list, JArr)) else i for i in idx)
    return idx


class _AtIdx:
    def __init__(self, arr, idx):
        self._arr = arr
        self._idx = _norm_idx(idx)

    def set(self, v):
        out = np.array(self._arr, copy=True).view(JArr)
        out[self._idx] = np.asarray(v)
        return out

    def add(self, v):
        out = np.array(self._arr, copy=True).view(JArr)
        np.add.at(out, self._idx, np.asarray(v))
        return out


def _wrap(x):
    if isinstance(x, np.ndarray) and not isinstance(x, JArr):
        return x.view(JArr)
    if isinstance(x, np.floating):  # jax returns 0-d arrays, not numpy scalars
        return np.asarray(x).view(JArr)
    if isinstance(x, tuple):
        return tuple(_wrap(i) for i in x)
    if isinstance(x, list):
        return [_wrap(i) for i in x]
    return x


def _wrapfn(fn):
    @functools.wraps(fn)
    def inner(*a, **k):
        return _wrap(fn(*a, **k))

    return inner


class _JnpModule(types.ModuleType):
    """``jax.numpy`` backed by numpy; array results come back as ``JArr``."""

    def __getattr__(self, name):
        obj = getattr(np, name)
        if callable(obj) and not isinstance(obj, type):
            return _wrapfn(obj)
        return obj


def _array(obj, dtype=None, **kw):
    return _wrap(np.array(obj, dtype=dtype))


def _jit(fun=None, **kwargs):
    if fun is None:
        return lambda f: f
    return fun


def _vmap(fun, in_axes=0, out_axes=0):
    def mapped(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        n = None
        for a, ax in zip(args, axes):
            if ax is not None:
                n = np.shape(a)[ax]
                break
        outs = []
        for i in range(n):
            call = [np.take(a, i, axis=ax) if ax is not None else a for a, ax in zip(args, axes)]
            outs.append(np.asarray(fun(*[_wrap(c) if isinstance(c, np.ndarray) else c for c in call])))
        return _wrap(np.stack(outs, axis=out_axes))

    return mapped


def _fori_loop(lo, hi, body, init):
    val = init
    for i in range(lo, hi):
        val = body(i, val)
    return val


def _while_loop(cond, body, init):
    val = init
    while bool(cond(val)):
        val = body(val)
    return val


def _tree_map(f, *trees):
    import dataclasses

    t0 = trees[0]
    if dataclasses.is_dataclass(t0):
        kw = {}
        for fld in dataclasses.fields(t0):
            kw[fld.name] = f(*[getattr(t, fld.name) for t in trees])
        return type(t0)(**kw)
    if isinstance(t0, tuple):
        return type(t0)(*[_tree_map(f, *xs) for xs in zip(*trees)])
    return f(*trees)


class _Comm:
    def Get_rank(self):
        return 0

    def Get_size(self):
        return 1


def install():
    """Register the shim modules (jax, jax.numpy, mpi4py, mpi4jax, matplotlib)."""
    jnp = _JnpModule("jax.numpy")
    jnp.array = _array
    jnp.asarray = _array
    jnp.ndarray = np.ndarray

    jax = types.ModuleType("jax")
    jax.numpy = jnp
    jax.jit = _jit
    jax.vmap = _vmap
    jax.Array = np.ndarray
    jax.device_get = lambda x: x
    jax.device_put = lambda x, *a, **k: x
    lax = types.ModuleType("jax.lax")
    lax.fori_loop = _fori_loop
    lax.while_loop = _while_loop
    jax.lax = lax
    tu = types.ModuleType("jax.tree_util")
    tu.register_pytree_node = lambda *a, **k: None
    tu.tree_map = _tree_map
    jax.tree_util = tu
    cfg = types.SimpleNamespace(update=lambda *a, **k: None)
    jax.config = cfg

    mpi4py = types.ModuleType("mpi4py")
    MPI = types.ModuleType("mpi4py.MPI")
    MPI.COMM_WORLD = _Comm()
    MPI.PROC_NULL = object()
    MPI.MIN = "min"
    MPI.MAX = "max"
    mpi4py.MPI = MPI

    mpi4jax = types.ModuleType("mpi4jax")
    mpi4jax.allreduce = lambda x, op=None, comm=None: x
    mpi4jax.sendrecv = lambda send, recv, source=None, dest=None, comm=None: recv

    mpl = types.ModuleType("matplotlib")
    plt = types.ModuleType("matplotlib.pyplot")
    mpl.pyplot = plt

    sys.modules.update(
        {
            "jax": jax,
            "jax.numpy": jnp,
            "jax.lax": lax,
            "jax.tree_util": tu,
            "mpi4py": mpi4py,
            "mpi4py.MPI": MPI,
            "mpi4jax": mpi4jax,
            "matplotlib": mpl,
            "matplotlib.pyplot": plt,
        }
    )
    return jax


def as_jarr(x):
    return np.asarray(x, dtype=np.float64).copy().view(JArr)
