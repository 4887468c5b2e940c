"""The CPU oracle against the golden vectors that the reference's own float64
code wrote (``tests/golden/make_golden.py``): the pin of every parity claim
of the kernels, which are checked against the oracle.

Tolerances: the reference's own float64 bar against LAL is a relative
error of 1e-10 and a mismatch of 1e-14 (its ``tests/test_xas.py:65-72``);
the oracle differs from the reference by rounding only (the fits expanded
into monomials, the closed-form collocation solutions solved as linear
systems), so it is held to 1e-11 on the waveforms and 1e-9 on the tables.
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import compare, golden
from oracle import phenomd, taylorf2, xas

MODELS = {"xas": ("IMRPhenomXAS", xas), "phenomd": ("IMRPhenomD", phenomd), "taylorf2": ("TaylorF2", taylorf2)}


@pytest.mark.parametrize("model", MODELS)
def test_cases(model):
    name, module = MODELS[model]
    g = golden(f"{model}_cases")
    hp, hc = oracle.polarizations(name, g["params"], g["frequencies"])
    for i in range(len(g["params"])):
        for a, b in ((hp[i], g["hplus"][i]), (hc[i], g["hcross"][i])):
            error, mismatch = compare(a, b)
            assert error < 1e-11, (i, error)
            assert mismatch < 1e-14, (i, mismatch)
    tables = module.flat(module.table(g["params"], g["frequencies"][:, 0]))
    ref = g["tables"]
    scale = np.maximum(np.abs(ref), 1e-300)
    assert np.all(np.where(ref != 0, np.abs(tables - ref) / scale, np.abs(tables)) < 1e-9)


@pytest.mark.parametrize("model", MODELS)
def test_single_workload(model):
    """The single binary on linspace(20, 1024, 4017) (the float64 workload)."""
    name, _ = MODELS[model]
    g = golden(f"{model}_cases")
    hp, hc = oracle.polarizations(name, g["single_params"], g["single_frequencies"])
    for a, b in ((hp[0], g["single_hplus"]), (hc[0], g["single_hcross"])):
        error, mismatch = compare(a, b)
        assert error < 1e-11 and mismatch < 1e-14


@pytest.mark.parametrize("model", MODELS)
@pytest.mark.parametrize("kind", ["random", "reference_mf", "unscaled"])
def test_other_fixtures(model, kind):
    name, _ = MODELS[model]
    g = golden(f"{model}_{kind}")
    kwargs = {}
    if kind == "reference_mf":
        kwargs["reference_mf"] = float(g["reference_mf"])
    if kind == "unscaled":
        kwargs["amp_scale"] = 1.0
    hp, hc = oracle.polarizations(name, g["params"], g["frequencies"], **kwargs)
    for a, b in ((hp, g["hplus"]), (hc, g["hcross"])):
        for i in range(len(a)):
            if np.all(np.isnan(b[i])):  # a binary the reference refuses
                assert np.all(np.isnan(a[i])), (kind, i)
                continue
            error, mismatch = compare(a[i], b[i])
            assert error < 1e-11 and mismatch < 1e-14, (kind, i, error)


def test_nan_where_lal_fails():
    g = golden("xas_nan")
    hp, hc = oracle.polarizations("IMRPhenomXAS", g["params"], g["frequencies"])
    assert np.all(np.isnan(hp)) and np.all(np.isnan(hc))
    assert np.all(np.isnan(g["hplus"]))


def test_taylorf2_binary_neutron_star():
    """A binary neutron star from 20 Hz (reference ``tests/test_taylorf2.py:97-109``):
    a leading phase term of about 10^4 radians."""
    g = golden("taylorf2_cases")
    hp, hc = oracle.polarizations("TaylorF2", g["bns_params"], g["bns_frequencies"])
    for a, b in ((hp[0], g["bns_hplus"]), (hc[0], g["bns_hcross"])):
        error, mismatch = compare(a, b)
        assert error < 1e-11 and mismatch < 1e-14


def test_taylorf2_reference_mf_refusal():
    """With ``reference_mf``, ``f_ref`` must be zero: NaN otherwise (the
    last binary of the fixture), as the reference."""
    g = golden("taylorf2_reference_mf")
    hp, _ = oracle.polarizations("TaylorF2", g["params"], g["frequencies"], reference_mf=float(g["reference_mf"]))
    assert np.all(np.isnan(hp[-1])) and np.all(np.isnan(g["hplus"][-1]))
    assert np.all(np.isfinite(hp[:-1]))


def test_qnm_fits():
    """The (2,2) QNM fits in powers of 1 - a: the reference's values exactly,
    and its direct fits to its rounding (reference ``tests/test_xas.py:142-154``)."""
    g = golden("qnm")
    values = np.array([xas.qnm(a) for a in g["spins"]])
    np.testing.assert_allclose(values, g["expanded"], rtol=1e-14)
    np.testing.assert_allclose(values, g["direct"], rtol=1e-10)


def test_t_c_extension():
    """``t_c`` multiplies the strain by exp(-2 pi i f t_c): a delay."""
    g = golden("xas_random")
    params, f = g["params"][:3], g["frequencies"]
    t_c = np.array([0.0, 0.05, -0.1])
    hp, hc = oracle.polarizations("IMRPhenomXAS", params, f, t_c=t_c)
    hp0, hc0 = oracle.polarizations("IMRPhenomXAS", params, f)
    np.testing.assert_allclose(hp, hp0 * np.exp(-2j * np.pi * f * t_c[:, None]), rtol=1e-13, atol=0)
    np.testing.assert_allclose(hc[0], hc0[0], rtol=0, atol=0)


def test_fd_gradient_of_loss_is_consistent():
    """Central differences of the oracle's loss at two steps agree (the
    gradient oracle of the kernels)."""
    g = golden("xas_random")
    params, f = g["params"][:2], g["frequencies"]
    w = 1.0 / oracle.api.psd(f)
    data = oracle.polarizations("IMRPhenomXAS", params * np.array([1.01, 0.99, 1, 1, 1, 1, 1, 1]), f)[0]
    g1 = oracle.loss_gradient_fd("IMRPhenomXAS", params, f, data, w, rel_step=1e-6)
    g2 = oracle.loss_gradient_fd("IMRPhenomXAS", params, f, data, w, rel_step=3e-6)
    assert np.all(np.abs(g1 - g2) <= 1e-5 * np.abs(g1) + 1e-7 * np.max(np.abs(g1), axis=1, keepdims=True))


def test_c_restatement_against_the_reference():
    """The oracle's C evaluation (oracle/xas_eval.c, the CPU baseline's) from
    the reference's own tables reproduces the reference's waveforms, and from
    the NumPy oracle's tables the NumPy oracle's, on shared and per-binary
    grids, with any number of threads."""
    from oracle import native, xas

    g = golden("xas_cases")
    for threads in (1, 3):
        hp, hc = native.xas_evaluate(g["tables"], g["frequencies"], threads)
        for a, b in ((hp, g["hplus"]), (hc, g["hcross"])):
            assert np.max(np.abs(a - b)) <= 1e-11 * np.max(np.abs(b))
    hp, hc = native.xas_evaluate(g["single_table"], g["single_frequencies"])
    assert np.max(np.abs(hp[0] - g["single_hplus"])) <= 1e-11 * np.max(np.abs(g["single_hplus"]))
    r = golden("xas_random")
    f = r["frequencies"] if "frequencies" in r else None
    params = r["params"]
    grid = np.linspace(20.0, 1024.0, 777) if f is None else f
    hp, hc = native.xas_polarizations(params, grid)
    ref_p, ref_c = xas.evaluate(xas.table(params, np.asarray(grid)[..., 0]), grid)
    ok = np.isfinite(ref_p)
    assert np.array_equal(ok, np.isfinite(hp))
    assert np.max(np.abs(hp[ok] - ref_p[ok])) <= 1e-11 * np.max(np.abs(ref_p[ok]))
    assert np.max(np.abs(hc[ok] - ref_c[ok])) <= 1e-11 * np.max(np.abs(ref_c[ok]))
