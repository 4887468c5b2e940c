"""The converters between LAL's reference convention (``Binary.f_ref`` in Hz)
and the mass-scaled one (``WaveformOptions.reference_mf``) for the models of
this path, as the reference's ``src/waveformx/_reference.py:59-80``
(``to_mass_scaled_reference``, ``to_physical_reference``, dispatching on
``approximant``).

For these aligned-spin models only ``phi_ref`` changes, by half the change
of the (2,2) phase between the two references
(``models/taylorf2/reference.py:46-104``): ``phi_ref' = phi_ref +
(Phi(f_2) - Phi(f_1)) / 2``, the change reduced modulo ``2 pi``
(IMRPhenomD, TaylorF2: ``phi_ref`` modulo ``pi``, the (2,2) unchanged) or
``4 pi`` (IMRPhenomXAS and IMRPhenomXHM, ``models/xas/reference.py:38``:
``phi_ref`` modulo ``2 pi``, every mode unchanged). ``f_ref = 0`` is the
first frequency ``f_min`` (NaN without it) for IMRPhenomD, IMRPhenomXAS and
IMRPhenomXHM, the reference at coalescence (no phase) for TaylorF2. The
phases ``Phi`` come from each model's FP64 set-up on the device
(``wfx_phase_difference``), one launch for a whole batch; the rest is a
vectorised host pass.
"""

from __future__ import annotations

import math

import numpy as np

from ._options import REFERENCE_MF
from .exceptions import KernelError, UnknownApproximantError, UnsupportedError

__all__ = ["REFERENCE_MODELS", "to_mass_scaled_reference", "to_physical_reference"]

MTSUN_SI = 4.925490947641267e-06

#: approximant -> (what f_ref = 0 means, the period of the phase change)
REFERENCE_MODELS = {
    "TaylorF2": ("coalescence", 2.0 * math.pi),
    "IMRPhenomD": ("f_min", 2.0 * math.pi),
    "IMRPhenomXAS": ("f_min", 4.0 * math.pi),
    "IMRPhenomXHM": ("f_min", 4.0 * math.pi),
}
_OTHER = ("IMRPhenomXPNR", "IMRPhenomXPNR_NNLO", "IMRPhenomXPNR_MSA", "NRSur7dq4")


def _model(approximant):
    if isinstance(approximant, str) and approximant in REFERENCE_MODELS:
        return REFERENCE_MODELS[approximant]
    if isinstance(approximant, str) and approximant in _OTHER:
        raise UnsupportedError(f"the converters of {approximant} are not on the aligned-spin B200 path "
                               f"({', '.join(REFERENCE_MODELS)})")
    raise UnknownApproximantError(f"unknown approximant {approximant!r}: waveformx_b200 implements "
                                  f"{', '.join(REFERENCE_MODELS)}")


def _numpy(value) -> np.ndarray:
    if hasattr(value, "detach"):
        return value.detach().cpu().numpy().astype(np.float64)
    return np.asarray(value, dtype=np.float64)


def _float32(binary) -> bool:
    """The binary's precision, as the reference's (FP32 iff every float
    field is float32)."""
    kinds = [str(getattr(v, "dtype", "float64")) for v in binary]
    return all(k in ("float32", "torch.float32") for k in kinds)


def _output(value: np.ndarray, template, float32: bool):
    """``value`` in the container of ``template``: a torch tensor on its
    device, a NumPy array, or a Python float."""
    if hasattr(template, "detach"):
        import torch

        return torch.as_tensor(np.array(value), dtype=torch.float32 if float32 else torch.float64,
                               device=template.device)
    out = np.asarray(value, dtype=np.float32 if float32 else np.float64)
    if out.ndim == 0 and not isinstance(template, np.ndarray):
        return out.item()
    return out


def _phase_change(approximant, binary, mf_from, mf_to) -> np.ndarray:
    """``Phi(mf_to) - Phi(mf_from)`` per binary, on the device."""
    import torch

    from . import _lib, ops

    model = ops.model_code(approximant)
    m1, m2 = _numpy(binary.mass_1), _numpy(binary.mass_2)
    chi1, chi2 = _numpy(binary.spin_1)[..., 2], _numpy(binary.spin_2)[..., 2]
    m1, m2, chi1, chi2, a, b = np.broadcast_arrays(m1, m2, chi1, chi2, mf_from, mf_to)
    shape = m1.shape
    n = max(1, m1.size)
    params = np.zeros((n, 8))
    for k, x in enumerate((m1, m2, chi1, chi2)):
        params[:, k] = x.reshape(-1)
    params[:, 4] = 1.0
    if not torch.cuda.is_available():
        raise KernelError("waveformx_b200 runs on a CUDA device and none is available")
    dev = torch.device("cuda", torch.cuda.current_device())
    p = torch.as_tensor(params, device=dev)
    ta = torch.as_tensor(np.ascontiguousarray(a.reshape(-1)), device=dev)
    tb = torch.as_tensor(np.ascontiguousarray(b.reshape(-1)), device=dev)
    out = torch.empty(n, dtype=torch.float64, device=dev)
    _lib.check("wfx_phase_difference", _lib.library().wfx_phase_difference(
        model, ops._ptr(p), n, ops._ptr(ta), ops._ptr(tb), ops._ptr(out), ops._stream(dev)))
    return out.cpu().numpy().reshape(shape)


def _mf(binary, f, zero_is, f_min) -> np.ndarray:
    """``M f`` at ``f`` (Hz): ``f = 0`` means ``f_min`` (NaN without it) or,
    at coalescence, no phase (0)."""
    total = _numpy(binary.mass_1) + _numpy(binary.mass_2)
    f = _numpy(f)
    if zero_is == "coalescence":
        return np.where(f > 0.0, f * total, 0.0) * MTSUN_SI
    f = np.where(f == 0.0, np.nan if f_min is None else _numpy(f_min), f)
    return np.where(f > 0.0, f, np.nan) * total * MTSUN_SI


def _shifted(binary, change: np.ndarray, period: float, f_ref):
    """``binary`` with ``phi_ref`` moved by half the change, reduced modulo
    the period, and ``f_ref`` replaced."""
    float32 = _float32(binary)
    turns = np.round(change / period)
    phi = _numpy(binary.phi_ref) + 0.5 * (change - turns * period)
    f_out = np.broadcast_to(_numpy(f_ref), phi.shape)
    return binary._replace(phi_ref=_output(phi, binary.phi_ref, float32),
                           f_ref=_output(f_out, binary.f_ref, float32))


def to_mass_scaled_reference(binary, reference_mf=REFERENCE_MF, f_min=None, *, approximant="IMRPhenomXPNR"):
    """``binary`` given at its reference frequency ``binary.f_ref`` (Hz,
    LAL's convention) as a binary given at the mass-scaled reference
    ``reference_mf / M`` (``f_ref`` zero), for ``approximant`` with
    ``WaveformOptions(reference_mf=reference_mf)``: only ``phi_ref``
    changes. ``f_min`` is the first frequency that ``f_ref = 0`` stands for
    (IMRPhenomD, IMRPhenomXAS, IMRPhenomXHM). ``approximant`` defaults to
    IMRPhenomXPNR, as the reference's, which is not on this path."""
    zero_is, period = _model(approximant)
    mf_from = _mf(binary, binary.f_ref, zero_is, f_min)
    change = _phase_change(approximant, binary, mf_from, float(reference_mf))
    return _shifted(binary, change, period, 0.0)


def to_physical_reference(binary, f_ref, reference_mf=REFERENCE_MF, *, approximant="IMRPhenomXPNR"):
    """The inverse of :func:`to_mass_scaled_reference`: ``binary`` given at
    the mass-scaled reference ``reference_mf / M`` (its ``f_ref`` ignored)
    as a binary given at ``f_ref`` (Hz, LAL's convention)."""
    zero_is, period = _model(approximant)
    mf_to = _mf(binary, f_ref, zero_is, None)
    change = _phase_change(approximant, binary, float(reference_mf), mf_to)
    return _shifted(binary, change, period, f_ref)
