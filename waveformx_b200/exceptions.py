"""The errors of waveformx_b200: the taxonomy of the reference
(``src/waveformx/exceptions.py``), so that code catching the reference's
errors catches these. Every error derives from :class:`WaveformError` and
from the matching built-in exception."""

__all__ = [
    "WaveformError",
    "InvalidParameterError",
    "UnsupportedError",
    "UnknownApproximantError",
    "ModelError",
    "KernelError",
]


class WaveformError(Exception):
    """Base class of the errors of waveformx_b200."""


class InvalidParameterError(WaveformError, ValueError):
    """A parameter that LALSimulation rejects for this approximant."""


class UnsupportedError(WaveformError, ValueError):
    """The approximant does not support the request."""


class UnknownApproximantError(WaveformError, ValueError):
    """The name is not an approximant of this path (IMRPhenomXAS, IMRPhenomD, TaylorF2)."""


class ModelError(WaveformError, RuntimeError):
    """The model could not be evaluated for this binary."""


class KernelError(WaveformError, RuntimeError):
    """A call of the CUDA library failed (its return code and message), or the
    library is missing where it must run."""
