"""The reference-convention converters on the device against the
reference's own (``tests/golden/converters.npz`` from
``models/{taylorf2,phenomd,xas}/reference.py``), and the property they
exist for: a binary converted to the mass-scaled reference gives, with
``reference_mf``, the same waveform as the original with its ``f_ref``
(``src/waveformx/_reference.py:8-16``)."""

from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu

MODELS = ("TaylorF2", "IMRPhenomD", "IMRPhenomXAS", "IMRPhenomXHM")


def _binary(params):
    import waveformx_b200 as wb

    p = params
    z = np.zeros(len(p))
    return wb.Binary(p[:, 0], p[:, 1], np.stack([z, z, p[:, 2]], -1), np.stack([z, z, p[:, 3]], -1), p[:, 4],
                     p[:, 5], p[:, 6], p[:, 7])


@pytest.mark.parametrize("model", MODELS)
def test_against_the_reference(cuda, model):
    import waveformx_b200 as wb

    data = golden("converters")
    key = "IMRPhenomXAS" if model == "IMRPhenomXHM" else model
    b = _binary(data["params"])
    scaled = wb.to_mass_scaled_reference(b, float(data["reference_mf"]), float(data["f_min"]), approximant=model)
    np.testing.assert_allclose(scaled.phi_ref, data[f"{key}_scaled_phi_ref"], rtol=0, atol=1e-9)
    assert np.all(np.asarray(scaled.f_ref) == 0.0)
    physical = wb.to_physical_reference(b, float(data["f_ref_out"]), float(data["reference_mf"]), approximant=model)
    np.testing.assert_allclose(physical.phi_ref, data[f"{key}_physical_phi_ref"], rtol=0, atol=1e-9)
    assert np.all(np.asarray(physical.f_ref) == float(data["f_ref_out"]))


@pytest.mark.parametrize("model", MODELS)
def test_round_trip(cuda, model):
    import waveformx_b200 as wb

    data = golden("converters")
    params = data["params"].copy()
    params[:, 7] = np.where(params[:, 7] == 0.0, 25.0, params[:, 7])
    b = _binary(params)
    back = wb.to_physical_reference(wb.to_mass_scaled_reference(b, 0.01, approximant=model), b.f_ref, 0.01,
                                    approximant=model)
    period = 2 * math.pi if model in ("IMRPhenomXAS", "IMRPhenomXHM") else math.pi
    d = (np.asarray(back.phi_ref) - b.phi_ref) / period
    np.testing.assert_allclose(d, np.round(d), atol=1e-9)


def test_one_binary_and_torch_fields(cuda):
    """A single binary of Python numbers stays numbers; torch fields stay
    tensors (float32 in, float32 out)."""
    import torch

    import waveformx_b200 as wb

    b = wb.Binary(36.0, 29.0, (0.0, 0.0, 0.3), (0.0, 0.0, -0.1), 500.0, 0.7, 1.2, 30.0)
    out = wb.to_mass_scaled_reference(b, 0.01, approximant="IMRPhenomXAS")
    assert isinstance(out.phi_ref, float) and out.f_ref == 0.0
    t = wb.Binary(*(torch.tensor(np.asarray(v, dtype=np.float32)) for v in b))
    out_t = wb.to_mass_scaled_reference(t, 0.01, approximant="IMRPhenomXAS")
    assert out_t.phi_ref.dtype == torch.float32
    assert float(out_t.phi_ref) == pytest.approx(out.phi_ref, abs=1e-5)


@pytest.mark.parametrize("model", ("IMRPhenomD", "IMRPhenomXAS", "IMRPhenomXHM"))
def test_same_waveform(cuda, model):
    """With reference_mf the converted binary gives the original waveform."""
    import torch

    import waveformx_b200 as wb
    from waveformx_b200 import _lib, ops

    data = golden("converters")
    params = data["params"][:6].copy()
    params[:, 7] = 30.0
    scaled = wb.to_mass_scaled_reference(_binary(params), 0.01, approximant=model)
    p2 = params.copy()
    p2[:, 6] = np.asarray(scaled.phi_ref)
    p2[:, 7] = 0.0
    f = torch.as_tensor(np.geomspace(20.0, 400.0, 300), device=cuda)
    outs = []
    for p, rmf in ((params, None), (p2, 0.01)):
        t = ops.setup(model, torch.as_tensor(p, device=cuda), f[:1], reference_mf=rmf, precision=_lib.FP64)
        outs.append(ops.polarizations(model, t.table, f)[0].cpu().numpy())
    a, r = outs
    assert np.max(np.abs(a - r)) / np.max(np.abs(r)) < 1e-8
