"""A NumPy stand-in for the small part of JAX that the reference's
aligned-spin frequency-domain modules touch, so that their own float64
arithmetic can run in a container without JAX to produce golden vectors.

Test infrastructure only: ``tests/golden/make_golden.py`` puts this
directory first on ``sys.path`` while it imports the reference's modules.
Nothing in the product imports it.

Transformations are identities (``jit``) or loops (``vmap``); ``jvp`` is
forward mode on dual numbers (exact derivatives, for the two derivatives
IMRPhenomXHM's set-up takes).
"""

from __future__ import annotations

import contextlib
import types

import numpy as _np

from . import lax, numpy, tree_util  # noqa: F401

__version__ = "0.0-numpy-shim"


class Array(_np.ndarray):
    """Never instantiated: ``isinstance(x, jax.Array)`` is False for every
    NumPy value, which makes the reference's optimisation barriers no-ops."""


class _Config:
    def update(self, *args, **kwargs):
        return None


config = _Config()


def jit(function=None, **kwargs):
    if function is None:
        return lambda f: f
    return function


def vmap(function, in_axes=0, out_axes=0):
    """A Python loop over the leading axis of the mapped arguments."""

    def mapped(*args):
        axes = in_axes if isinstance(in_axes, (tuple, list)) else (in_axes,) * len(args)
        n = None
        for a, ax in zip(args, axes):
            if ax is not None:
                n = len(tree_util.tree_leaves(a)[0])
                break
        outs = []
        for i in range(n):
            call = [tree_util.tree_map(lambda x: x[i], a) if ax is not None else a for a, ax in zip(args, axes)]
            outs.append(function(*call))
        return tree_util.tree_map(lambda *xs: _np.stack(xs), *outs)

    return mapped


@contextlib.contextmanager
def ensure_compile_time_eval():
    yield


class ShapeDtypeStruct(types.SimpleNamespace):
    def __init__(self, shape, dtype):
        super().__init__(shape=shape, dtype=dtype)


class _Dual(_np.lib.mixins.NDArrayOperatorsMixin):
    """A value and its tangent (forward mode), for :func:`jvp`: NumPy's
    ufuncs and the few array functions the reference's set-up applies to
    them carry the tangent by the chain rule; comparisons give plain
    arrays."""

    __array_priority__ = 1000

    def __init__(self, value, tangent):
        # (the parts may be duals themselves: a derivative of a derivative)
        self.v = value if isinstance(value, _Dual) else _np.asarray(value)
        if isinstance(tangent, _Dual):
            self.d = tangent
        elif isinstance(self.v, _Dual):
            self.d = _np.asarray(tangent, dtype=float)
        else:
            self.d = _np.broadcast_to(_np.asarray(tangent, dtype=self.v.dtype), self.v.shape).copy()

    @property
    def shape(self):
        return _np.shape(self.v)

    @property
    def ndim(self):
        return _np.ndim(self.v)

    @property
    def dtype(self):
        return self.v.dtype

    def __getitem__(self, index):
        return _Dual(self.v[index], self.d[index])

    def reshape(self, *shape):
        return _Dual(self.v.reshape(*shape), self.d.reshape(*shape))

    def astype(self, dtype):
        return _Dual(self.v.astype(dtype), self.d.astype(dtype))

    def __float__(self):
        return float(self.v)

    def __array_ufunc__(self, ufunc, method, *inputs, **kwargs):
        if method != "__call__" or kwargs.get("out") is not None:
            return NotImplemented
        vs = [x.v if isinstance(x, _Dual) else _np.asarray(x) for x in inputs]
        ds = [x.d if isinstance(x, _Dual) else _np.zeros(_np.shape(x)) for x in inputs]
        name = ufunc.__name__
        if name in _PLAIN:
            return ufunc(*vs)
        value = ufunc(*vs)
        rule = _RULES.get(name)
        if rule is None:
            raise NotImplementedError(f"jvp of {name} in the shim")
        return _Dual(value, rule(value, vs, ds))

    def __array_function__(self, func, types, args, kwargs):
        name = func.__name__
        if name == "where":
            cond, a, b = args
            cond = cond.v if isinstance(cond, _Dual) else cond
            av, ad = (a.v, a.d) if isinstance(a, _Dual) else (_np.asarray(a), 0.0)
            bv, bd = (b.v, b.d) if isinstance(b, _Dual) else (_np.asarray(b), 0.0)
            while isinstance(cond, _Dual):
                cond = cond.v
            return _Dual(_np.where(cond, av, bv), _np.where(cond, ad, bd))
        if name == "clip":
            x, lo, hi = args
            inside = (x.v >= lo) & (x.v <= hi)
            return _Dual(_np.clip(x.v, lo, hi), _np.where(inside, x.d, 0.0))
        if name in ("stack", "concatenate"):
            seq = args[0]
            vs = [s.v if isinstance(s, _Dual) else _np.asarray(s) for s in seq]
            ds = [s.d if isinstance(s, _Dual) else _np.zeros_like(_np.asarray(s, dtype=float)) for s in seq]
            return _Dual(func(vs, *args[1:], **kwargs), func(ds, *args[1:], **kwargs))
        if name in ("broadcast_to", "expand_dims", "squeeze", "moveaxis", "transpose"):
            x = args[0]
            return _Dual(func(x.v, *args[1:], **kwargs), func(x.d, *args[1:], **kwargs))
        if name in ("shape", "ndim", "result_type", "isnan", "isfinite", "isinf", "signbit", "ones_like",
                    "zeros_like", "full_like"):
            plain = [a.v if isinstance(a, _Dual) else a for a in args]
            return func(*plain, **kwargs)
        if name == "sum":
            x = args[0]
            return _Dual(_np.sum(x.v, *args[1:], **kwargs), _np.sum(x.d, *args[1:], **kwargs))
        raise NotImplementedError(f"jvp through {name} in the shim")


_PLAIN = {"less", "less_equal", "greater", "greater_equal", "equal", "not_equal", "isnan", "isfinite", "isinf",
          "signbit", "logical_and", "logical_or", "logical_not", "sign", "floor", "ceil", "rint", "trunc"}


def _pow_rule(value, vs, ds):
    a, b = vs
    da, db = ds
    with _np.errstate(divide="ignore", invalid="ignore"):
        out = b * _np.power(a, b - 1.0) * da
        if _np.any(db != 0):
            out = out + value * _np.log(a) * db
    return out


_RULES = {
    "add": lambda r, v, d: d[0] + d[1],
    "subtract": lambda r, v, d: d[0] - d[1],
    "multiply": lambda r, v, d: d[0] * v[1] + v[0] * d[1],
    "divide": lambda r, v, d: (d[0] - r * d[1]) / v[1],
    "true_divide": lambda r, v, d: (d[0] - r * d[1]) / v[1],
    "negative": lambda r, v, d: -d[0],
    "positive": lambda r, v, d: d[0],
    "power": _pow_rule,
    "float_power": _pow_rule,
    "square": lambda r, v, d: 2.0 * v[0] * d[0],
    "reciprocal": lambda r, v, d: -r * r * d[0],
    "exp": lambda r, v, d: r * d[0],
    "expm1": lambda r, v, d: (r + 1.0) * d[0],
    "log": lambda r, v, d: d[0] / v[0],
    "log1p": lambda r, v, d: d[0] / (1.0 + v[0]),
    "sqrt": lambda r, v, d: 0.5 * d[0] / r,
    "cbrt": lambda r, v, d: d[0] / (3.0 * r * r),
    "sin": lambda r, v, d: _np.cos(v[0]) * d[0],
    "cos": lambda r, v, d: -_np.sin(v[0]) * d[0],
    "tan": lambda r, v, d: (1.0 + r * r) * d[0],
    "tanh": lambda r, v, d: (1.0 - r * r) * d[0],
    "arctan": lambda r, v, d: d[0] / (1.0 + v[0] * v[0]),
    "arctan2": lambda r, v, d: (v[1] * d[0] - v[0] * d[1]) / (v[0] * v[0] + v[1] * v[1]),
    "hypot": lambda r, v, d: (v[0] * d[0] + v[1] * d[1]) / r,
    "absolute": lambda r, v, d: _np.where(v[0] < 0, -d[0], d[0]),
    "maximum": lambda r, v, d: _np.where(v[0] >= v[1], d[0], d[1]),
    "minimum": lambda r, v, d: _np.where(v[0] <= v[1], d[0], d[1]),
}


def jvp(function, primals, tangents):
    """``(function(*primals), its derivative along tangents)`` by forward
    mode (:class:`_Dual`)."""
    out = function(*[_Dual(p, t) for p, t in zip(primals, tangents)])
    if isinstance(out, _Dual):
        return out.v, out.d
    return out, _np.zeros_like(_np.asarray(out, dtype=float))
