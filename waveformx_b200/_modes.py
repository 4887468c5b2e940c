"""The single-binary calls of the reference's API with keyword parameters:
``polarizations`` and ``polarizations_on_grid`` (``src/waveformx/
_api.py:156-177``), and the modes in the conventions of
``SimInspiralChooseFDModes``,
as the reference's ``modes`` and ``choose_fd_modes`` (``src/waveformx/
_api.py:180-204``): of the models of this path only IMRPhenomXHM has them
(``models/xhm/api.py:75-116``); IMRPhenomXAS, IMRPhenomD and TaylorF2
raise ``UnsupportedError`` as the reference's do.

The modes ``h_{l,-m}`` at the positive frequencies come from the kernels
(``ops.xhm_modes``, FP64); the two-sided layout is host-side:
``h_{l,m}(-f) = (-1)^l conj(h_{l,-m}(f))`` at the negative frequencies,
zero at the other half (``models/xhm/api.py:38-50``).
"""

from __future__ import annotations

import math
from dataclasses import dataclass
from typing import Any, Dict, Optional, Tuple

import numpy as np

from ._binary import BINARY_NAMES, Binary, check_binary
from ._options import WaveformOptions, parse_options, strain_scale
from ._results import check_frequencies
from .exceptions import InvalidParameterError, UnknownApproximantError, UnsupportedError

__all__ = ["FrequencyModes", "binary_from_keywords", "modes", "choose_fd_modes", "polarizations_from_modes",
           "polarizations", "polarizations_on_grid"]

Mode = Tuple[int, int]
MTSUN_SI = 4.925490947641267e-06
_ALIGNED = ("IMRPhenomXAS", "IMRPhenomD", "TaylorF2")


@dataclass
class FrequencyModes:
    """Modes ``h_lm`` in the conventions of ``SimInspiralChooseFDModes``
    (the reference's ``_results.py:72-97``): ``frequencies`` (two-sided)
    and a dict ``{(l, m): array}``, with the angles ``theta`` and ``phi`` of
    the line of sight in the frame of the modes and the
    ``polarization_angle`` that rotates their polarizations into LAL's."""

    frequencies: Any
    modes: Dict[Mode, Any]
    theta: float = 0.0
    phi: float = 0.0
    polarization_angle: float = 0.0

    def __getitem__(self, mode: Mode):
        return self.modes[tuple(mode)]

    def __iter__(self):
        return iter((self.frequencies, self.modes))

    def polarizations(self):
        """``(h_+, h_x)`` on the non-negative frequencies from the modes,
        summed with the spin-weighted spherical harmonics at ``(theta,
        phi)`` and rotated by the polarization angle."""
        return polarizations_from_modes(self)


def _wigner_d(ell: int, mp: int, m: int, beta: float) -> float:
    """Wigner's ``d^l_{m' m}(beta)`` (LAL's ``XLALWignerdMatrix``
    convention)."""
    f = math.factorial
    ch, sh = math.cos(beta / 2), math.sin(beta / 2)
    pre = math.sqrt(f(ell + mp) * f(ell - mp) * f(ell + m) * f(ell - m))
    total = 0.0
    for k in range(max(0, m - mp), min(ell + m, ell - mp) + 1):
        c = (-1) ** (k - m + mp) * pre / (f(ell + m - k) * f(k) * f(ell - k - mp) * f(k - m + mp))
        total += c * ch ** (2 * ell - 2 * k + m - mp) * sh ** (2 * k - m + mp)
    return total


def _ylm(theta: float, phi: float, ell: int, m: int) -> complex:
    """``{-2}Y_{lm}(theta, phi)`` (``XLALSpinWeightedSphericalHarmonic``)."""
    return math.sqrt((2 * ell + 1) / (4 * math.pi)) * _wigner_d(ell, m, 2, theta) * complex(math.cos(m * phi),
                                                                                          math.sin(m * phi))


def polarizations_from_modes(fm: FrequencyModes):
    """``(h_+, h_x)`` on the non-negative frequencies of two-sided modes:
    ``h_+ = 1/2 sum (h_lm(f) Y + conj(h_lm(-f) Y))``, ``h_x = i/2 sum
    (h_lm(f) Y - conj(h_lm(-f) Y))``, rotated by twice the polarization
    angle (the reference's ``_harmonics.py:39-67``)."""
    frequencies = np.asarray(fm.frequencies)
    n2 = frequencies.shape[0]
    n = int(np.sum(frequencies >= 0))
    hp = np.zeros(n, dtype=np.complex128)
    hc = np.zeros(n, dtype=np.complex128)
    for (ell, m), h in fm.modes.items():
        h = np.asarray(h)
        positive = h[n2 - n:]
        negative = h[:n][::-1]
        y = _ylm(fm.theta, fm.phi, ell, m)
        a = positive * y
        b = np.conj(negative) * np.conj(y)
        hp = hp + 0.5 * (a + b)
        hc = hc + 0.5j * (a - b)
    c, s = math.cos(2 * fm.polarization_angle), math.sin(2 * fm.polarization_angle)
    return hp * c + hc * s, hc * c - hp * s


def binary_from_keywords(keywords: Dict[str, Any]) -> Binary:
    """The binary of keyword arguments (``mass_1``, ``mass_2`` required),
    as the reference's ``_binary.py:83-105``: ``TypeError`` for unknown or
    missing names."""
    unknown = [name for name in keywords if name not in BINARY_NAMES]
    if unknown:
        raise TypeError(f"unexpected keyword argument {unknown[0]!r}: the binary parameters are "
                        f"{', '.join(BINARY_NAMES)}")
    for name in ("mass_1", "mass_2"):
        if name not in keywords:
            raise TypeError(f"missing required keyword argument {name!r}")
    values = {}
    for name in BINARY_NAMES:
        default = (0.0, 0.0, 0.0) if name in ("spin_1", "spin_2") else Binary._field_defaults.get(name)
        value = np.asarray(keywords.get(name, default), dtype=np.float64)
        if name in ("spin_1", "spin_2"):
            if value.shape != (3,):
                raise ValueError(f"{name} must have three components")
        elif value.ndim != 0:
            raise ValueError(f"{name} must be a scalar")
        values[name] = value if value.ndim else float(value)
    return Binary(**values)


def _request(options: Optional[WaveformOptions], keywords: Dict[str, Any]):
    binary = binary_from_keywords({k: v for k, v in keywords.items() if k in BINARY_NAMES})
    options = parse_options(options, {k: v for k, v in keywords.items() if k not in BINARY_NAMES})
    check_binary(binary)
    return binary, options


def _check_approximant(approximant: str) -> None:
    if approximant == "IMRPhenomXHM":
        return
    if approximant in _ALIGNED:
        raise UnsupportedError(f"the modes of {approximant} are not implemented in waveformx")
    from . import ops

    ops.model_code(approximant)  # (unknown, or off this path)
    raise UnsupportedError(f"the modes of {approximant} are not on the B200 path")


def _xhm_modes(binary: Binary, frequencies: np.ndarray, options: WaveformOptions) -> Dict[Mode, np.ndarray]:
    """The modes ``{(l, m): h_{l,-m}(f)}`` (m > 0) at the frequencies on the
    kernels (FP64), after the model's checks (``models/xhm/api.py:66-72``)."""
    import torch

    from . import _lib, ops
    from ._batch import status_errors

    if options.mode_array is not None:
        raise UnsupportedError("IMRPhenomXHM computes every mode: select them from modes()")
    if options.reference_mf is not None and float(binary.f_ref) != 0.0:
        raise InvalidParameterError("with reference_mf, the reference frequency is reference_mf / M: f_ref must be "
                                    "zero (to_mass_scaled_reference converts a binary given at f_ref)")
    if not torch.cuda.is_available():
        from .exceptions import KernelError

        raise KernelError("waveformx_b200 runs on a CUDA device and none is available")
    dev = torch.device("cuda", torch.cuda.current_device())
    p = torch.tensor([[float(binary.mass_1), float(binary.mass_2), float(np.asarray(binary.spin_1)[2]),
                       float(np.asarray(binary.spin_2)[2]), float(binary.luminosity_distance),
                       float(binary.inclination), float(binary.phi_ref), float(binary.f_ref)]],
                     dtype=torch.float64, device=dev)
    f = torch.as_tensor(np.asarray(frequencies, dtype=np.float64), device=dev)
    tables = ops.setup("IMRPhenomXHM", p, f[:1], amp_scale=strain_scale(options), reference_mf=options.reference_mf,
                       precision=_lib.FP64)
    errors = status_errors(tables.status.cpu().numpy(), "IMRPhenomXHM")
    if errors:
        raise errors[0]
    _, _, out = ops.xhm_modes(tables.table, f)
    out = out.cpu().numpy()[0]
    return {mode: out[k] for k, mode in enumerate(ops.XHM_MODES)}


def _two_sided(one_sided: Dict[Mode, np.ndarray], frequencies: np.ndarray, inclination: float) -> FrequencyModes:
    """``h_{l,-m}`` at the positive frequencies, ``h_{l,m}(-f) = (-1)^l
    conj(h_{l,-m}(f))`` at the negative ones (``models/xhm/api.py:38-50``)."""
    zero = np.zeros_like(one_sided[(2, 2)])
    out = {}
    for (ell, emm), h in one_sided.items():
        sign = -1.0 if ell % 2 else 1.0
        out[(ell, -emm)] = np.concatenate([zero, h])
        out[(ell, emm)] = np.concatenate([(sign * np.conj(h))[::-1], zero])
    two_sided = np.concatenate([-frequencies[::-1], frequencies])
    return FrequencyModes(two_sided, dict(sorted(out.items())), float(inclination), math.pi / 2, 0.0)


def modes(approximant: str, frequencies: Any, *, options: Optional[WaveformOptions] = None,
          **keywords) -> FrequencyModes:
    """The modes ``h_lm`` at ``+-frequencies`` (``SimInspiralChooseFDModes``
    conventions) of the binary given by the keywords (the reference's
    ``modes``, ``_api.py:180-187``); IMRPhenomXHM only, as the reference."""
    _check_approximant(approximant)
    binary, options = _request(options, keywords)
    frequencies = check_frequencies(frequencies)
    one = _xhm_modes(binary, frequencies, options)
    return _two_sided(one, np.asarray(frequencies, dtype=np.float64), float(binary.inclination))


def choose_fd_modes(approximant: str, delta_f: float, f_min: float, f_max: float = 0.0, *,
                    options: Optional[WaveformOptions] = None, **keywords) -> FrequencyModes:
    """``SimInspiralChooseFDModes`` (the reference's ``_api.py:190-204``,
    ``models/xhm/api.py:83-116``): the modes on LAL's two-sided uniform grid
    ``k delta_f``, zero below ``f_min`` and above ``min(f_max, f_cut)``,
    ``f_ref = 0`` meaning ``f_min``."""
    _check_approximant(approximant)
    binary, options = _request(options, keywords)
    if not delta_f > 0 or not f_min > 0 or f_max < 0:
        raise InvalidParameterError("delta_f and f_min must be positive and f_max non-negative")
    m1, m2 = float(binary.mass_1), float(binary.mass_2)
    chi1, chi2 = float(np.asarray(binary.spin_1)[2]), float(np.asarray(binary.spin_2)[2])
    if m1 < m2:
        m1, m2, chi1, chi2 = m2, m1, chi2, chi1
    eta = m1 * m2 / (m1 + m2) ** 2
    delta = math.sqrt(max(1.0 - 4.0 * eta, 0.0))
    chi_eff = 0.5 * (1.0 + delta) * chi1 + 0.5 * (1.0 - delta) * chi2
    f_cut = (0.33 if chi_eff > 0.99 else 0.3) / ((m1 + m2) * MTSUN_SI)
    f_max_prime = min(f_max if f_max != 0.0 else f_cut, f_cut)
    i_start = int(f_min / delta_f)
    i_stop = int(f_max_prime / delta_f) + 1
    last = f_max if f_max_prime < f_max else f_max_prime
    n_full = int(2.0 ** np.ceil(np.log2(int(last / delta_f)))) + 1
    n = max(n_full, i_stop)
    if float(binary.f_ref) == 0.0 and options.reference_mf is None:
        binary = binary._replace(f_ref=float(f_min))
    band = np.arange(i_start, i_stop) * delta_f
    one = _xhm_modes(binary, band, options)
    full = {}
    for mode, h in one.items():
        # (the one-mode functions vanish above f_max_prime)
        padded = np.zeros(n, dtype=np.complex128)
        padded[i_start:i_stop] = h
        full[mode] = padded[:n_full]
    frequencies = np.arange(n_full) * delta_f
    two = _two_sided(full, frequencies, float(binary.inclination))
    # (a zero frequency appears once)
    keep = np.r_[np.arange(n_full - 1), np.arange(n_full, 2 * n_full)]
    return FrequencyModes(two.frequencies[keep], {k: v[keep] for k, v in two.modes.items()}, two.theta, two.phi, 0.0)


def polarizations(approximant: str, frequencies: Any, *, options: Optional[WaveformOptions] = None, **keywords):
    """``(h_+, h_x)`` of the binary given by the keywords at ``frequencies``
    (Hz), as ``SimInspiralChooseFDWaveformSequence`` (the reference's
    ``polarizations``, ``_api.py:156-170``): the model's checks first
    (``InvalidParameterError``), then the FP64 kernels; complex128 NumPy
    arrays."""
    import torch

    from . import _lib, ops
    from ._batch import status_errors

    ops.model_code(approximant)
    binary, options = _request(options, keywords)
    frequencies = check_frequencies(frequencies)
    if options.reference_mf is not None and float(binary.f_ref) != 0.0:
        raise InvalidParameterError("with reference_mf, the reference frequency is reference_mf / M: f_ref must be "
                                    "zero (to_mass_scaled_reference converts a binary given at f_ref)")
    if not torch.cuda.is_available():
        from .exceptions import KernelError

        raise KernelError("waveformx_b200 runs on a CUDA device and none is available")
    dev = torch.device("cuda", torch.cuda.current_device())
    p = torch.tensor([[float(binary.mass_1), float(binary.mass_2), float(np.asarray(binary.spin_1)[2]),
                       float(np.asarray(binary.spin_2)[2]), float(binary.luminosity_distance),
                       float(binary.inclination), float(binary.phi_ref), float(binary.f_ref)]],
                     dtype=torch.float64, device=dev)
    if np.any(np.asarray(binary.spin_1)[:2] != 0) or np.any(np.asarray(binary.spin_2)[:2] != 0):
        raise InvalidParameterError(f"non-zero in-plane spins were given, but {approximant} is a non-precessing "
                                    "approximant")
    f = torch.as_tensor(np.asarray(frequencies, dtype=np.float64), device=dev)
    tables = ops.setup(approximant, p, f[:1], amp_scale=strain_scale(options), reference_mf=options.reference_mf,
                       precision=_lib.FP64)
    errors = status_errors(tables.status.cpu().numpy(), approximant)
    if errors:
        raise errors[0]
    hp, hc = ops.polarizations(approximant, tables.table, f)
    return hp.cpu().numpy()[0], hc.cpu().numpy()[0]


def polarizations_on_grid(approximant: str, grid: Any, *, options: Optional[WaveformOptions] = None, **keywords):
    """``(h_+, h_x)`` on a :class:`FrequencyGrid` (or frequencies), as the
    reference's ``polarizations_on_grid`` (``_api.py:173-177``)."""
    from ._results import FrequencyGrid

    frequencies = grid.frequencies if isinstance(grid, FrequencyGrid) else grid
    return polarizations(approximant, frequencies, options=options, **keywords)
