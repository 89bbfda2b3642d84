"""NumPy stand-in for ``jax``, ``jax.numpy`` and ``opt_einsum``.

Used ONLY by ``make_golden.py`` to execute the reference's own tenax source
(loaded by file path from a read-only checkout) with float64 NumPy arithmetic
so that golden input/output fixtures can be generated in a container that has
no jax/jaxlib.  Nothing in the product package, the oracle, the GPU tests or
the benchmark imports this module.

What is emulated:
  * ``jnp.*``: numpy functions whose array results are viewed as ``_JArr``,
    an ndarray subclass with the functional ``.at[idx].set/.add`` API.
  * ``jax.random``: a deterministic key -> numpy Generator mapping
    (values differ from real JAX; fixtures store the generated inputs).
  * ``jax.tree_util.register_pytree_node_class``, ``jax.jit``,
    ``jax.lax.stop_gradient``: identity (optionally recording its argument,
    see ``record_stop_gradient``).
  * ``jax.lax.while_loop / fori_loop / cond / scan``: eager Python loops.
  * ``opt_einsum.contract_expression / contract / contract_path``:
    ``np.einsum`` with a path computed once per expression.
"""

from __future__ import annotations

import sys
import types

import numpy as np


class _AtHelper:
    def __init__(self, arr, idx):
        self._arr = arr
        self._idx = idx

    def set(self, value):
        out = np.array(self._arr, copy=True).view(_JArr)
        out[self._idx] = value
        return out

    def add(self, value):
        out = np.array(self._arr, copy=True).view(_JArr)
        np.add.at(out, self._idx, value)
        return out

    def multiply(self, value):
        out = np.array(self._arr, copy=True).view(_JArr)
        out[self._idx] = out[self._idx] * value
        return out

    def get(self):
        return self._arr[self._idx]


class _AtIndexer:
    def __init__(self, arr):
        self._arr = arr

    def __getitem__(self, idx):
        return _AtHelper(self._arr, idx)


class _JArr(np.ndarray):
    @property
    def at(self):
        return _AtIndexer(self)

    def block_until_ready(self):
        return self


def _wrap(x):
    if isinstance(x, np.ndarray) and not isinstance(x, _JArr):
        return x.view(_JArr)
    if isinstance(x, tuple):
        return tuple(_wrap(v) for v in x)
    if isinstance(x, list):
        return [_wrap(v) for v in x]
    return x


def _wrapped(fn):
    def inner(*args, **kwargs):
        return _wrap(fn(*args, **kwargs))

    inner.__name__ = getattr(fn, "__name__", "fn")
    return inner


class _NumpyModule(types.ModuleType):
    """Module whose attributes are numpy's, with array results wrapped."""

    def __init__(self, name, base):
        super().__init__(name)
        self._base = base

    def __getattr__(self, item):
        val = getattr(self._base, item)
        if callable(val) and not isinstance(val, type):
            return _wrapped(val)
        return val


def _array(x, dtype=None, copy=True):
    return np.array(x, dtype=dtype).view(_JArr)


_SG_LOG = None


def record_stop_gradient(log) -> None:
    """Append a copy of every array passed to ``jax.lax.stop_gradient`` to
    ``log`` (a list), or stop recording when ``log`` is None.  The CTM moves
    of algorithms/ipeps.py pass exactly their projectors through it."""
    global _SG_LOG
    _SG_LOG = log


_SVD_LOG = None


def record_svd(log) -> None:
    """Append (U, s, Vh) of every ``jnp.linalg.svd(..., compute_uv=True)``
    call to ``log``, or stop recording when ``log`` is None."""
    global _SVD_LOG
    _SVD_LOG = log


def install() -> None:
    """Register the stand-in modules in ``sys.modules``."""
    jnp = _NumpyModule("jax.numpy", np)
    jnp.array = _array
    jnp.asarray = _array

    def einsum(subscripts, *operands, optimize=True, **kwargs):
        # jnp.einsum contracts pairwise along an optimised path by default
        return _wrap(np.einsum(subscripts, *operands, optimize=optimize, **kwargs))

    jnp.einsum = einsum
    jnp.float64 = np.float64
    jnp.float32 = np.float32
    jnp.complex128 = np.complex128
    jnp.complex64 = np.complex64
    jnp.int32 = np.int32
    jnp.ndarray = np.ndarray
    jnp.linalg = _NumpyModule("jax.numpy.linalg", np.linalg)

    def svd(a, full_matrices=True, compute_uv=True, **kw):
        r = np.linalg.svd(np.asarray(a), full_matrices=full_matrices, compute_uv=compute_uv)
        if compute_uv and _SVD_LOG is not None:
            _SVD_LOG.append(tuple(np.array(x, dtype=np.float64, copy=True) for x in r))
        return _wrap(tuple(r) if compute_uv else r)

    jnp.linalg.svd = svd

    jax = types.ModuleType("jax")
    jax.numpy = jnp
    jax.Array = np.ndarray

    class _Config:
        def update(self, *a, **k):
            return None

    jax.config = _Config()

    def jit(fn=None, **kwargs):
        if fn is None:
            return lambda f: f
        return fn

    jax.jit = jit
    jax.vmap = lambda f, *a, **k: f
    jax.block_until_ready = lambda x: x

    tree_util = types.ModuleType("jax.tree_util")
    tree_util.register_pytree_node_class = lambda cls: cls
    tree_util.tree_map = lambda f, *t: f(*t)
    jax.tree_util = tree_util

    core = types.ModuleType("jax.core")

    class Tracer:  # never instantiated
        pass

    core.Tracer = Tracer
    jax.core = core

    lax = types.ModuleType("jax.lax")
    def stop_gradient(x):
        if _SG_LOG is not None:
            _SG_LOG.append(np.array(x, dtype=np.float64, copy=True))
        return x

    lax.stop_gradient = stop_gradient

    def while_loop(cond_fun, body_fun, init_val):
        val = init_val
        while bool(cond_fun(val)):
            val = body_fun(val)
        return val

    def fori_loop(lower, upper, body_fun, init_val):
        val = init_val
        for i in range(int(lower), int(upper)):
            val = body_fun(i, val)
        return val

    def cond(pred, true_fun, false_fun, *operands):
        return true_fun(*operands) if bool(pred) else false_fun(*operands)

    def dynamic_update_slice(operand, update, start_indices):
        # start indices are clamped so that the update fits, as in XLA
        out = np.array(operand, copy=True)
        upd = np.asarray(update)
        sl = []
        for s, n, m in zip(start_indices, out.shape, upd.shape):
            s = min(max(int(s), 0), n - m)
            sl.append(slice(s, s + m))
        out[tuple(sl)] = upd
        return out.view(_JArr)

    lax.dynamic_update_slice = dynamic_update_slice
    lax.while_loop = while_loop
    lax.fori_loop = fori_loop
    lax.cond = cond
    jax.lax = lax

    random = types.ModuleType("jax.random")

    def PRNGKey(seed):
        return np.array([0, int(seed) & 0xFFFFFFFF], dtype=np.uint32)

    def fold_in(key, data):
        k = np.asarray(key, dtype=np.uint64)
        mixed = (int(k[1]) * 0x9E3779B1 + int(data) * 0x85EBCA77 + int(k[0])) & 0xFFFFFFFF
        return np.array([int(k[1]) & 0xFFFFFFFF, mixed], dtype=np.uint32)

    def split(key, num=2):
        return np.stack([fold_in(key, 1000003 + i) for i in range(num)])

    def _gen(key):
        k = np.asarray(key, dtype=np.uint64)
        return np.random.default_rng([int(k[0]), int(k[1])])

    def normal(key, shape=(), dtype=np.float64):
        return _gen(key).standard_normal(shape).astype(dtype).view(_JArr)

    def uniform(key, shape=(), dtype=np.float64, minval=0.0, maxval=1.0):
        return _gen(key).uniform(minval, maxval, shape).astype(dtype).view(_JArr)

    random.PRNGKey = PRNGKey
    random.key = PRNGKey
    random.fold_in = fold_in
    random.split = split
    random.normal = normal
    random.uniform = uniform
    jax.random = random

    oe = types.ModuleType("opt_einsum")

    class _Expr:
        def __init__(self, subscripts, shapes):
            self.subscripts = subscripts
            dummies = [np.empty(s) for s in shapes]
            self.path = np.einsum_path(subscripts, *dummies, optimize="optimal")[0]

        def __call__(self, *arrays, backend=None):
            return _wrap(np.einsum(self.subscripts, *arrays, optimize=self.path))

    def contract_expression(subscripts, *shapes, optimize="auto"):
        return _Expr(subscripts, shapes)

    def contract(subscripts, *arrays, optimize="auto", backend=None):
        return _wrap(np.einsum(subscripts, *arrays, optimize=True))

    class _PathInfo:
        def __init__(self, path):
            self.path = path

    def contract_path(subscripts, *arrays, optimize="auto"):
        path = np.einsum_path(subscripts, *arrays, optimize="optimal")[0]
        return path, _PathInfo(path[1:])

    oe.contract_expression = contract_expression
    oe.contract = contract
    oe.contract_path = contract_path

    sys.modules["jax"] = jax
    sys.modules["jax.numpy"] = jnp
    sys.modules["jax.numpy.linalg"] = jnp.linalg
    sys.modules["jax.tree_util"] = tree_util
    sys.modules["jax.core"] = core
    sys.modules["jax.lax"] = lax
    sys.modules["jax.random"] = random
    sys.modules["opt_einsum"] = oe


def load_reference(src_root: str, modules: list[str]) -> dict[str, types.ModuleType]:
    """Import reference modules by file path without running tenax/__init__.py.

    ``src_root`` is the directory that contains the ``tenax`` package.
    Parent packages are created as empty namespace modules so that
    ``from tenax.core.index import ...`` inside the reference resolves.
    """
    import importlib
    import os

    install()
    pkgs = ["tenax", "tenax.core", "tenax.contraction", "tenax.network", "tenax.algorithms"]
    for p in pkgs:
        if p in sys.modules:
            continue
        m = types.ModuleType(p)
        m.__path__ = [os.path.join(src_root, *p.split("."))]
        sys.modules[p] = m
    core_pkg = sys.modules["tenax.core"]
    if not hasattr(core_pkg, "EPS"):
        # tenax/core/__init__.py only re-exports the core modules and defines
        # the EPS constants that algorithms/ipeps.py imports from it.
        path = os.path.join(src_root, "tenax", "core", "__init__.py")
        with open(path) as fh:
            exec(compile(fh.read(), path, "exec"), core_pkg.__dict__)
    out = {}
    for name in modules:
        out[name] = importlib.import_module(name)
    return out
