"""``jax.lax`` for the NumPy shim: the few primitives the reference's
aligned-spin modules call."""

import numpy as np


def stop_gradient(x):
    return x


def optimization_barrier(x):
    return x


def complex(re, im):  # noqa: A001 (the name of jax.lax.complex)
    return np.asarray(re) + 1j * np.asarray(im)
