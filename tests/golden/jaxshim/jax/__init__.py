"""A NumPy stand-in for the small part of JAX that the reference's
aligned-spin frequency-domain modules touch, so that their own float64
arithmetic can run in a container without JAX to produce golden vectors.

Test infrastructure only: ``tests/golden/make_golden.py`` puts this
directory first on ``sys.path`` while it imports the reference's modules.
Nothing in the product imports it.

Transformations are identities (``jit``) or loops (``vmap``); there is no
differentiation.
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
