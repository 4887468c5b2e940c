"""``batch_polarizations``: the reference's batch function
(``src/waveformx/_api.py:307-360``, its ``tests/test_xas.py:103-121``):
batch equals single, failed binaries reported in ``ok``/``errors`` and
zeroed, ``strict`` raising the first error, chunking, ragged grids."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import golden

pytestmark = pytest.mark.gpu


def _table(params):
    t = np.zeros((len(params), 12))
    t[:, [0, 1, 4, 7, 8, 9, 10, 11]] = params
    return t


@pytest.mark.parametrize("approximant,model",
                         [("IMRPhenomXAS", "xas"), ("IMRPhenomD", "phenomd"), ("TaylorF2", "taylorf2")])
def test_batch_equals_golden(cuda, approximant, model):
    import waveformx_b200 as wb

    g = golden(f"{model}_random")
    out = wb.batch_polarizations(approximant, g["frequencies"], _table(g["params"]), chunk_size=7)
    assert out.ok.all() and not out.errors
    assert out.hplus.dtype.is_complex and out.hplus.shape == g["hplus"].shape
    for a, b in ((out.hplus, g["hplus"]), (out.hcross, g["hcross"])):
        a = a.cpu().numpy()
        np.testing.assert_allclose(a, b, rtol=1e-10, atol=1e-10 * np.abs(b).max())


def test_failures_and_strict(cuda):
    import torch

    import waveformx_b200 as wb

    g = golden("xas_random")
    table = _table(g["params"][:5])
    table[1, 0] = -3.0                    # a negative mass: the common checks
    table[2, 2] = 0.2                     # an in-plane spin
    table[3, :2] = [2000.0, 1.0]          # a mass ratio beyond 1000: the set-up's status
    out = wb.batch_polarizations("IMRPhenomXAS", g["frequencies"], table)
    assert list(out.ok) == [True, False, False, False, True]
    assert isinstance(out.errors[1], wb.InvalidParameterError) and "positive" in str(out.errors[1])
    assert "in-plane" in str(out.errors[2])
    assert "1000" in str(out.errors[3])
    assert torch.all(out.hplus[1:4] == 0)
    ref = oracle.polarizations("IMRPhenomXAS", g["params"][[0, 4]], g["frequencies"])[0]
    np.testing.assert_allclose(out.hplus[[0, 4]].cpu().numpy(), ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max())
    with pytest.raises(wb.InvalidParameterError, match="positive"):
        wb.batch_polarizations("IMRPhenomXAS", g["frequencies"], table, strict=True)
    # numpy output and float32
    out = wb.batch_polarizations("IMRPhenomXAS", g["frequencies"], table[[0, 4]], output="numpy",
                                 dtype=torch.float32)
    assert isinstance(out.hplus, np.ndarray) and out.hplus.dtype == np.complex64


def test_ragged_batch(cuda):
    import torch

    import waveformx_b200 as wb

    g = golden("xas_cases")
    table = _table(g["params"])
    grids = [x[: 100 + 7 * i] for i, x in enumerate(g["frequencies"])]
    out = wb.batch_polarizations("IMRPhenomXAS", grids, table, dtype=torch.float32)
    assert out.ok.all()
    for i, (hp, grid) in enumerate(zip(out.hplus, grids)):
        ref = oracle.polarizations("IMRPhenomXAS", g["params"][i:i + 1].astype(np.float32).astype(np.float64),
                                   grid.astype(np.float32).astype(np.float64))[0][0]
        assert hp.shape == (len(grid),)
        assert oracle.mismatch(hp.cpu().numpy(), ref) < 1e-6


def test_taylorf2_checks(cuda):
    """TaylorF2's own checks (reference ``models/taylorf2/api.py:44-49``):
    no in-plane spins, and f_ref zero with ``reference_mf``; f_ref = 0 is the
    reference at coalescence."""
    import waveformx_b200 as wb

    g = golden("taylorf2_random")
    table = _table(g["params"][:4])
    table[1, 5] = 0.1                     # an in-plane spin
    table[3, 11] = 0.0                    # the reference at coalescence
    out = wb.batch_polarizations("TaylorF2", g["frequencies"], table)
    assert list(out.ok) == [True, False, True, True]
    assert "in-plane" in str(out.errors[1])
    params = g["params"][:4].copy()
    params[3, 7] = 0.0
    ref = oracle.polarizations("TaylorF2", params[[0, 2, 3]], g["frequencies"])[0]
    np.testing.assert_allclose(out.hplus[[0, 2, 3]].cpu().numpy(), ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max())
    out = wb.batch_polarizations("TaylorF2", g["frequencies"], table[[0, 3]], reference_mf=0.01)
    assert list(out.ok) == [False, True]
    assert "f_ref must be zero" in str(out.errors[0])
    ref = oracle.polarizations("TaylorF2", params[[3]], g["frequencies"], reference_mf=0.01)[0]
    np.testing.assert_allclose(out.hplus[1].cpu().numpy(), ref[0], rtol=1e-10, atol=1e-10 * np.abs(ref).max())


def test_empty_batch(cuda):
    """No binaries: empty results, as the reference's (its zeros of shape
    (0, N) and an empty ok)."""
    import torch

    import waveformx_b200 as wb

    f = np.linspace(20.0, 512.0, 101)
    for dtype in (torch.float64, torch.float32):
        out = wb.batch_polarizations("IMRPhenomXAS", f, np.zeros((0, 12)), dtype=dtype)
        assert tuple(out.hplus.shape) == (0, 101) and tuple(out.hcross.shape) == (0, 101)
        assert out.ok.shape == (0,) and not out.errors
        out = wb.batch_polarizations("IMRPhenomXAS", [], np.zeros((0, 12)), dtype=dtype)
        assert out.ok.shape == (0,) and not out.errors


@pytest.mark.parametrize("approximant", ["IMRPhenomXAS", "IMRPhenomD", "TaylorF2", "IMRPhenomXHM"])
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
def test_ragged_with_empty_rows(cuda, approximant, precision):
    """Ragged batches with binaries of no frequency (first, middle, last) and
    of one: each non-empty row equals that binary alone on its own grid; the
    empty rows are empty."""
    import torch

    import waveformx_b200 as wb

    dtype = torch.float32 if precision == "fp32" else torch.float64
    g = golden("xas_cases")
    table = _table(g["params"][:7])
    base = g["frequencies"][0]
    grids = [base[:0], base[:300], base[:0], base[10:11], base[5:700], base[:123], base[:0]]
    out = wb.batch_polarizations(approximant, grids, table, dtype=dtype)
    for i, grid in enumerate(grids):
        assert tuple(out.hplus[i].shape) == (len(grid),) and tuple(out.hcross[i].shape) == (len(grid),)
        if not len(grid):
            continue
        single = wb.batch_polarizations(approximant, [grid], table[i:i + 1], dtype=dtype)
        assert out.ok[i] == single.ok[0]
        # (the same evaluation; the FP32 kernel may group the frequencies of
        # a row differently at another offset of the flat grid)
        tol = 1e-6 if precision == "fp32" else 1e-12
        for a, b in ((out.hplus[i], single.hplus[0]), (out.hcross[i], single.hcross[0])):
            a, b = a.cpu().numpy(), b.cpu().numpy()
            np.testing.assert_allclose(a, b, rtol=0, atol=tol * np.abs(b).max())
