"""The FP64 per-binary set-up kernel against the reference's golden tables,
and its dual-number derivatives against central differences of itself.

Tolerances: the set-up restates the reference's float64 arithmetic with the
device's math functions (cbrt, log, exp, pow, atan within an ulp of the
host's) and Gaussian elimination for the collocation systems; the tables
agree to 1e-8 relative (the worst entries are coefficients formed by
cancellation, which are the same waveforms to 1e-13).
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden
from layouts import reference_flat, relative_error

pytestmark = pytest.mark.gpu

MODELS = {"xas": "IMRPhenomXAS", "phenomd": "IMRPhenomD", "taylorf2": "TaylorF2"}


def _setup(cuda, approximant, params, f_min, amp_scale=1e21, reference_mf=None, precision=0, jvp=False):
    import torch

    from waveformx_b200 import ops

    p = torch.as_tensor(np.asarray(params, dtype=np.float64), device=cuda)
    f = torch.as_tensor(np.asarray(f_min, dtype=np.float64), device=cuda)
    return ops.setup(approximant, p, f, amp_scale=amp_scale, reference_mf=reference_mf, precision=precision, jvp=jvp)


@pytest.mark.parametrize("model", MODELS)
@pytest.mark.parametrize("kind", ["cases", "random", "reference_mf", "unscaled"])
def test_tables_match_golden(cuda, model, kind):
    g = golden(f"{model}_{kind}")
    f = g["frequencies"]
    f_min = f[:, 0] if f.ndim == 2 else np.full(len(g["params"]), f[0])
    kwargs = {}
    if kind == "reference_mf":
        kwargs["reference_mf"] = float(g["reference_mf"])
    if kind == "unscaled":
        kwargs["amp_scale"] = 1.0
    tables = _setup(cuda, MODELS[model], g["params"], f_min, **kwargs)
    ours = reference_flat(model, tables.table.cpu().numpy())
    ref = g["tables"]
    used = np.any(ref != 0, axis=0)
    # (a binary the reference refuses has NaN where LAL fails: the same
    # entries are NaN here, and its status is set)
    np.testing.assert_array_equal(np.isnan(ours[:, used]), np.isnan(ref[:, used]))
    assert relative_error(ours[:, used], ref[:, used]) < 1e-8
    refused = np.any(np.isnan(ref), axis=1)
    status = tables.status.cpu().numpy()
    assert np.all(status[~refused] == 0) and np.all(status[refused] != 0)


def test_status_where_lal_refuses(cuda):
    bad = np.array([[2000.0, 1.0, 0.0, 0.0, 400.0, 0.4, 0.0, 20.0],   # mass ratio
                    [36.0, 29.0, 0.3, -0.1, 500.0, 0.7, 1.2, 20.0],   # fine
                    [36.0, -29.0, 0.3, -0.1, 500.0, 0.7, 1.2, 20.0]])  # negative mass
    tables = _setup(cuda, "IMRPhenomXAS", bad, np.full(3, 20.0))
    status = tables.status.cpu().numpy()
    assert status[0] & 1 and status[1] == 0 and status[2] & 64
    tab = tables.table.cpu().numpy()
    assert np.isnan(tab[0, 54]) and np.isfinite(tab[1, 54])
    # reference_mf with a non-zero f_ref
    tables = _setup(cuda, "IMRPhenomD", bad[1:2], [20.0], reference_mf=0.01)
    assert tables.status.cpu().numpy()[0] & 32


@pytest.mark.parametrize("model", MODELS)
def test_jvp_matches_central_differences(cuda, model):
    g = golden(f"{model}_random")
    params = g["params"][:6].copy()
    params[:, 7] = 25.0
    f_min = np.full(len(params), 20.0)
    tables = _setup(cuda, MODELS[model], params, f_min, jvp=True)
    d = tables.dtable.cpu().numpy()
    value = _setup(cuda, MODELS[model], params, f_min).table.cpu().numpy()
    # (the set-up is compiled without FMA contraction: the dual numbers'
    # values round as the plain set-up's)
    np.testing.assert_array_equal(tables.table.cpu().numpy(), value)
    for k in range(8):
        h = 1e-6 * np.maximum(np.abs(params[:, k]), 1.0)
        up, down = params.copy(), params.copy()
        up[:, k] += h
        down[:, k] -= h
        fd = (_setup(cuda, MODELS[model], up, f_min).table.cpu().numpy()
              - _setup(cuda, MODELS[model], down, f_min).table.cpu().numpy()) / (2 * h[:, None])
        scale = np.abs(fd).max(axis=1, keepdims=True)
        err = np.abs(fd - d[:, :, k]) / (np.abs(fd) + 1e-6 * scale + 1e-300)
        assert err.max() < 1e-3, (k, err.max())


@pytest.mark.parametrize("model", MODELS)
def test_jvp_same_in_small_and_large_batches(cuda, model):
    """The dual-number set-up gives the same bits for the same binaries in a
    batch of 16 and in one of 2100 (every chain its own, whatever the
    blocks around it: amplitude and phase parts on different blocks for
    IMRPhenomXAS and IMRPhenomD, whole chains for TaylorF2)."""
    rng = np.random.default_rng(11)
    g = golden(f"{model}_random")
    params = g["params"][rng.integers(0, len(g["params"]), 2100)].copy()
    params[:, 7] = rng.choice([0.0, 20.0, 30.0], len(params))
    big = _setup(cuda, MODELS[model], params, np.full(len(params), 20.0), jvp=True)
    for lo in (0, 1000, 2084):
        small = _setup(cuda, MODELS[model], params[lo:lo + 16], np.full(16, 20.0), jvp=True)
        for a, b in ((small.table, big.table), (small.dtable, big.dtable), (small.status, big.status)):
            np.testing.assert_array_equal(a.cpu().numpy(), b[lo:lo + 16].cpu().numpy())
