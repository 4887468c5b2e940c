"""``WaveformOptions``: the settings the models take, with the fields,
defaults and checks of the reference's (``src/waveformx/_options.py:75-185``).

The aligned-spin path honours ``scaled_strain`` (the strain times
:data:`STRAIN_SCALE`) and ``reference_mf`` (a mass-scaled reference
frequency); ``precession_version``, ``mode_array`` and
``extended_phase_grid`` are accepted and checked as the reference does, and
do not change IMRPhenomXAS, IMRPhenomD or TaylorF2.
"""

from __future__ import annotations

import dataclasses
from typing import Any, Mapping, Optional, Tuple

from .exceptions import InvalidParameterError

__all__ = ["WaveformOptions", "OPTION_NAMES", "REFERENCE_MF", "STRAIN_SCALE", "parse_options", "strain_scale"]

#: The recommended ``reference_mf`` (late in every binary's inspiral).
REFERENCE_MF = 0.01
#: The factor of the strain unless ``scaled_strain`` is false: it keeps the
#: strain and its square inside the range of float32.
STRAIN_SCALE = 1e21

_PRECESSION_NAMES = {"nnlo": 102, "msa": 223, "spintaylor": 320, "spin_taylor": 320}


def _check_precession_version(value: Any) -> int:
    if isinstance(value, str):
        if value.lower() not in _PRECESSION_NAMES:
            raise InvalidParameterError(
                f"unknown precession version {value!r}: use 102 (\"NNLO\"), 223 (\"MSA\") or 320 (\"SpinTaylor\")")
        return _PRECESSION_NAMES[value.lower()]
    if isinstance(value, bool) or not isinstance(value, int):
        raise TypeError("precession_version must be an int (LAL's PhenomXPrecVersion) or a str")
    if value not in (102, 223, 320):
        raise InvalidParameterError(
            f"precession version {value} is not implemented: use 102 (NNLO), 223 (MSA) or 320 (SpinTaylor)")
    return value


def _check_mode_array(value: Any) -> Optional[Tuple[Tuple[int, int], ...]]:
    if value is None:
        return None
    if isinstance(value, str):
        raise TypeError("mode_array must be a sequence of (l, m) pairs or None")
    out = []
    for pair in value:
        try:
            ell, emm = (int(x) for x in pair)
        except (TypeError, ValueError):
            raise TypeError("mode_array must be a sequence of (l, m) pairs or None") from None
        out.append((ell, emm))
    return tuple(out)


def _check_reference_mf(value: Any) -> Optional[float]:
    if value is None:
        return None
    if isinstance(value, bool):
        raise TypeError("reference_mf must be a float or None")
    try:
        value = float(value)
    except (TypeError, ValueError):
        raise TypeError("reference_mf must be a float or None") from None
    if not 0.0 < value < 0.015:
        raise InvalidParameterError(
            f"reference_mf = {value} must lie in (0, 0.015): the inspiral of some binaries ends at M f = 0.015")
    return value


def _check_bool(value: Any, name: str) -> bool:
    if not isinstance(value, bool):
        raise TypeError(f"{name} must be a bool")
    return value


@dataclasses.dataclass(frozen=True)
class WaveformOptions:
    """The settings of LALSimulation's ``LALDict`` the models take: immutable
    and hashable (cache keys of the compiled functions).

    * ``precession_version`` (102, 223 or 320, or their names),
      ``mode_array`` and ``extended_phase_grid``: checked, unused by the
      aligned-spin models;
    * ``scaled_strain``: the strain times ``1e21`` (default ``True``);
    * ``reference_mf``: the reference frequency as ``M f_ref`` (default
      ``None``: ``Binary.f_ref`` in Hz); ``Binary.f_ref`` must then be zero
      (the waveform is NaN otherwise).
    """

    precession_version: int = 320
    mode_array: Optional[Tuple[Tuple[int, int], ...]] = None
    extended_phase_grid: bool = False
    scaled_strain: bool = True
    reference_mf: Optional[float] = None

    def __post_init__(self):
        object.__setattr__(self, "precession_version", _check_precession_version(self.precession_version))
        object.__setattr__(self, "mode_array", _check_mode_array(self.mode_array))
        _check_bool(self.extended_phase_grid, "extended_phase_grid")
        _check_bool(self.scaled_strain, "scaled_strain")
        object.__setattr__(self, "reference_mf", _check_reference_mf(self.reference_mf))

    @staticmethod
    def lalsimulation_defaults() -> "WaveformOptions":
        """LALSimulation's defaults for an empty ``LALDict`` (the strain
        itself, not scaled)."""
        return WaveformOptions(precession_version=223, scaled_strain=False)

    def replace(self, **options: Any) -> "WaveformOptions":
        """A copy with the given options changed."""
        _check_names(options)
        return dataclasses.replace(self, **options)

    def as_dict(self) -> dict:
        return {f.name: getattr(self, f.name) for f in dataclasses.fields(self)}


OPTION_NAMES = tuple(f.name for f in dataclasses.fields(WaveformOptions))


def strain_scale(options: WaveformOptions) -> float:
    """:data:`STRAIN_SCALE` if ``options.scaled_strain``, else 1."""
    return STRAIN_SCALE if options.scaled_strain else 1.0


def _check_names(options) -> None:
    for name in options:
        if name not in OPTION_NAMES:
            raise TypeError(f"unexpected keyword argument {name!r}: the options are {', '.join(OPTION_NAMES)}")


def parse_options(options: Optional[WaveformOptions], keywords: Mapping[str, Any]) -> WaveformOptions:
    """``options`` (default ``WaveformOptions()``) with ``keywords`` applied."""
    if options is None:
        options = WaveformOptions()
    elif not isinstance(options, WaveformOptions):
        raise TypeError("options must be a WaveformOptions or None")
    return options.replace(**keywords) if keywords else options
