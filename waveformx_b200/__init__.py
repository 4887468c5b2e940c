"""waveformx_b200: the aligned-spin frequency-domain path of waveformx
(IMRPhenomXAS, IMRPhenomD and TaylorF2 polarizations of batches of binaries,
and IMRPhenomXHM's modes and polarizations) on
hand-written sm_100a CUDA kernels behind a C ABI (``include/waveformx_b200.h``).

The Python interface is the reference's for this path:

* :func:`waveformx_b200.torch.polarizations_function` — the drop-in for
  ``waveformx.torch.polarizations_function`` (autograd through the backward
  kernel; ``t_c`` extension);
* :func:`batch_polarizations` — the drop-in for
  ``waveformx.batch_polarizations`` (same checks, ``ok``/``errors``,
  chunking; ragged batches; FP32 or FP64);
* :func:`polarizations`, :func:`polarizations_on_grid` — one binary by
  keywords, as the reference's;
* :func:`modes`, :func:`choose_fd_modes` — IMRPhenomXHM's modes in the
  conventions of ``SimInspiralChooseFDModes`` (:class:`FrequencyModes`);
* :func:`to_mass_scaled_reference`, :func:`to_physical_reference` — the
  converters between LAL's reference convention and the mass-scaled one;
* :mod:`waveformx_b200.ops` — tensor-level calls of the kernels: the
  per-binary tables, the polarizations, their vector-Jacobian product and
  the fused likelihood with its gradient.

Importing the package does not import torch; the CUDA library loads on first
use and every entry raises :class:`KernelError` without it or without a
CUDA device (there is no CPU fallback).
"""

from ._binary import BINARY_NAMES, COLUMNS, Binary, check_binary, parameter_table  # noqa: F401
from ._options import OPTION_NAMES, REFERENCE_MF, STRAIN_SCALE, WaveformOptions, parse_options  # noqa: F401
from ._results import BatchPolarizations, FrequencyGrid, check_frequencies  # noqa: F401
from .exceptions import (  # noqa: F401
    InvalidParameterError,
    KernelError,
    ModelError,
    UnknownApproximantError,
    UnsupportedError,
    WaveformError,
)

__version__ = "0.1.0"

__all__ = [
    "Binary", "BINARY_NAMES", "COLUMNS", "parameter_table", "check_binary", "WaveformOptions", "OPTION_NAMES",
    "REFERENCE_MF", "STRAIN_SCALE", "parse_options", "FrequencyGrid", "BatchPolarizations", "check_frequencies",
    "WaveformError", "InvalidParameterError", "UnsupportedError", "UnknownApproximantError", "ModelError",
    "KernelError", "approximants", "batch_polarizations", "polarizations_function", "to_mass_scaled_reference",
    "to_physical_reference", "modes", "choose_fd_modes", "FrequencyModes", "polarizations", "polarizations_on_grid",
]


def approximants(domain=None) -> list:
    """The approximants of this path (all frequency-domain)."""
    if domain not in (None, "frequency", "time"):
        raise ValueError('domain must be None, "frequency" or "time"')
    return [] if domain == "time" else ["IMRPhenomD", "IMRPhenomXAS", "IMRPhenomXHM", "TaylorF2"]


def batch_polarizations(approximant, grid, parameters, **keywords):
    """See :func:`waveformx_b200._batch.batch_polarizations`."""
    from ._batch import batch_polarizations as _batch

    return _batch(approximant, grid, parameters, **keywords)


def __getattr__(name):
    # (the modes' module imports the kernels' wrappers lazily)
    if name == "FrequencyModes":
        from ._modes import FrequencyModes

        return FrequencyModes
    raise AttributeError(name)


def polarizations(approximant, frequencies, *, options=None, **keywords):
    """See :func:`waveformx_b200._modes.polarizations`."""
    from ._modes import polarizations as _polarizations

    return _polarizations(approximant, frequencies, options=options, **keywords)


def polarizations_on_grid(approximant, grid, *, options=None, **keywords):
    """See :func:`waveformx_b200._modes.polarizations_on_grid`."""
    from ._modes import polarizations_on_grid as _on_grid

    return _on_grid(approximant, grid, options=options, **keywords)


def modes(approximant, frequencies, *, options=None, **keywords):
    """See :func:`waveformx_b200._modes.modes`."""
    from ._modes import modes as _modes

    return _modes(approximant, frequencies, options=options, **keywords)


def choose_fd_modes(approximant, delta_f, f_min, f_max=0.0, *, options=None, **keywords):
    """See :func:`waveformx_b200._modes.choose_fd_modes`."""
    from ._modes import choose_fd_modes as _choose

    return _choose(approximant, delta_f, f_min, f_max, options=options, **keywords)


def to_mass_scaled_reference(binary, reference_mf=REFERENCE_MF, f_min=None, *, approximant="IMRPhenomXPNR"):
    """See :func:`waveformx_b200._reference.to_mass_scaled_reference`."""
    from ._reference import to_mass_scaled_reference as _convert

    return _convert(binary, reference_mf, f_min, approximant=approximant)


def to_physical_reference(binary, f_ref, reference_mf=REFERENCE_MF, *, approximant="IMRPhenomXPNR"):
    """See :func:`waveformx_b200._reference.to_physical_reference`."""
    from ._reference import to_physical_reference as _convert

    return _convert(binary, f_ref, reference_mf, approximant=approximant)


def polarizations_function(approximant, options=None, **option_keywords):
    """The PyTorch function of :func:`waveformx_b200.torch.polarizations_function`."""
    from .torch import polarizations_function as _function

    return _function(approximant, options, **option_keywords)
