"""``jax.numpy.linalg`` for the NumPy shim (LAPACK's LU solve, as JAX's
CPU backend)."""

from numpy.linalg import solve  # noqa: F401
