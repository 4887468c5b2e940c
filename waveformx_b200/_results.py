"""Frequency grids and batch results, with the attributes of the
reference's (``src/waveformx/_results.py:31-170``)."""

from __future__ import annotations

import dataclasses
from typing import Any, Dict

import numpy as np

from .exceptions import InvalidParameterError

__all__ = ["FrequencyGrid", "BatchPolarizations", "check_frequencies"]


def check_frequencies(frequencies: Any) -> np.ndarray:
    """``frequencies`` as a 1-d float64 array, checked to be positive, finite
    and strictly increasing."""
    values = np.asarray(frequencies, dtype=float)
    if values.ndim != 1:
        raise InvalidParameterError("frequencies must be a 1-d array")
    if values.size and (not np.all(np.isfinite(values)) or values[0] <= 0):
        raise InvalidParameterError("frequencies must be positive and finite")
    if np.any(np.diff(values) <= 0):
        raise InvalidParameterError("frequencies must be strictly increasing")
    return values


class FrequencyGrid:
    """Frequencies (Hz) shared by many waveforms."""

    def __init__(self, frequencies: Any):
        self._frequencies = check_frequencies(frequencies)

    @staticmethod
    def uniform(f_min: float, f_max: float, delta_f: float) -> "FrequencyGrid":
        """``f_min, f_min + delta_f, ...`` up to ``f_max`` (within half a step)."""
        n = int(np.floor((f_max - f_min) / delta_f + 0.5)) + 1
        return FrequencyGrid(f_min + np.arange(n) * delta_f)

    @property
    def frequencies(self) -> np.ndarray:
        return self._frequencies

    def __len__(self) -> int:
        return int(self._frequencies.shape[0])

    def __repr__(self) -> str:
        f = self._frequencies
        lo, hi = (float(f[0]), float(f[-1])) if len(self) else (0.0, 0.0)
        return f"FrequencyGrid({len(self)} frequencies, {lo:g}-{hi:g} Hz)"


@dataclasses.dataclass
class BatchPolarizations:
    """``(n_binaries, n_frequencies)`` ``hplus`` and ``hcross`` (torch
    tensors on the device, or numpy arrays; lists of 1-d rows for a ragged
    batch), with ``ok`` (whether each binary succeeded) and ``errors``
    (``{index: exception}``); failed rows are zero."""

    hplus: Any
    hcross: Any
    ok: np.ndarray
    errors: Dict[int, Exception]

    def __iter__(self):
        return iter((self.hplus, self.hcross))
