"""The host logic of the Python layer, without a GPU: the parameter table,
the vectorised checks (the reference's per-row validation), the options,
the status words, the registry."""

from __future__ import annotations

import numpy as np
import pytest

import waveformx_b200 as wb
from waveformx_b200._batch import status_errors
from waveformx_b200._binary import aligned_table, table_errors


def test_parameter_table_forms():
    rows = {"mass_1": [36.0, 50.0], "mass_2": [29.0, 2.0], "spin_1": [[0, 0, 0.3], [0, 0, 0.9]],
            "spin_2z": [-0.4, 0.3], "f_ref": [20.0, 0.0]}
    t = wb.parameter_table(rows)
    assert t.shape == (2, 12)
    assert t[0, 4] == 0.3 and t[1, 7] == 0.3 and t[0, 8] == 1.0 and t[1, 11] == 0.0
    structured = np.zeros(2, dtype=[(c, float) for c in wb.COLUMNS])
    structured["mass_1"] = [1.0, 2.0]
    structured["mass_2"] = [1.0, 1.0]
    assert wb.parameter_table(structured).shape == (2, 12)
    np.testing.assert_array_equal(wb.parameter_table(t), t)
    with pytest.raises(TypeError, match="mass_2"):
        wb.parameter_table({"mass_1": [1.0]})
    with pytest.raises(TypeError, match="unknown"):
        wb.parameter_table({"mass_1": [1.0], "mass_2": [1.0], "mass_3": [1.0]})
    with pytest.raises(ValueError, match="12 columns"):
        wb.parameter_table(np.zeros((2, 5)))
    np.testing.assert_array_equal(aligned_table(t)[0], [36.0, 29.0, 0.3, -0.4, 1.0, 0.0, 0.0, 20.0])


def test_vectorised_checks_match_the_reference_rules():
    good = [36.0, 29.0, 0, 0, 0.3, 0, 0, -0.4, 500.0, 0.7, 1.2, 20.0]
    table = np.array([good] * 8)
    table[1, 0] = -1.0
    table[2, 4] = 1.5
    table[3, 8] = 0.0
    table[4, 11] = -2.0
    table[5, 9] = np.nan
    table[6, 3] = 0.1
    errors = table_errors(table, "IMRPhenomXAS")
    assert sorted(errors) == [1, 2, 3, 4, 5, 6]
    assert all(isinstance(e, wb.InvalidParameterError) for e in errors.values())
    assert "positive" in str(errors[1]) and "spin_1" in str(errors[2]) and "distance" in str(errors[3])
    assert "f_ref" in str(errors[4]) and "inclination" in str(errors[5]) and "in-plane" in str(errors[6])
    with pytest.raises(wb.InvalidParameterError):
        wb.check_binary(wb.Binary(-1.0, 29.0, (0, 0, 0), (0, 0, 0)))
    wb.check_binary(wb.Binary(36.0, 29.0, (0, 0, 0.3), (0, 0, 0)))


def test_status_words():
    errors = status_errors(np.array([0, 1, 8, 16 | 4, 32]), "IMRPhenomXAS")
    assert sorted(errors) == [1, 2, 3, 4]
    assert "1000" in str(errors[1]) and "final spin" in str(errors[2]) and "final mass" in str(errors[3])
    assert "reference_mf" in str(errors[4])
    assert "IMRPhenomD" in str(status_errors(np.array([8]), "IMRPhenomD")[0])


def test_options():
    o = wb.WaveformOptions()
    assert o.scaled_strain and o.reference_mf is None and o.precession_version == 320
    assert wb.WaveformOptions(precession_version="MSA").precession_version == 223
    assert wb.parse_options(None, {"scaled_strain": False}).scaled_strain is False
    with pytest.raises(wb.InvalidParameterError):
        wb.WaveformOptions(reference_mf=0.5)
    with pytest.raises(TypeError):
        wb.WaveformOptions(scaled_strain=1)
    with pytest.raises(TypeError, match="unexpected"):
        o.replace(colour="red")
    assert hash(o) == hash(wb.WaveformOptions())
    assert wb.WaveformOptions.lalsimulation_defaults().scaled_strain is False


def test_registry_and_grids():
    from waveformx_b200 import ops

    assert ops.model_code("IMRPhenomXAS") == 0 and ops.model_code("IMRPhenomD") == 1
    assert ops.model_code("TaylorF2") == 2
    with pytest.raises(wb.UnsupportedError):
        ops.model_code("IMRPhenomXPNR")
    with pytest.raises(wb.UnknownApproximantError):
        ops.model_code("nope")
    assert wb.approximants() == ["IMRPhenomD", "IMRPhenomXAS", "IMRPhenomXHM", "TaylorF2"] and wb.approximants("time") == []
    g = wb.FrequencyGrid.uniform(20.0, 30.0, 0.25)
    assert len(g) == 41 and g.frequencies[-1] == 30.0
    with pytest.raises(wb.InvalidParameterError):
        wb.FrequencyGrid([20.0, 19.0])


def test_converters_dispatch():
    """The converters' approximant: the reference's default (IMRPhenomXPNR)
    is off this path, an unknown name is an error; both before any device
    work."""
    b = wb.Binary(30.0, 20.0, (0, 0, 0.1), (0, 0, 0.2), 400.0, 0.3, 0.5, 20.0)
    with pytest.raises(wb.UnsupportedError):
        wb.to_mass_scaled_reference(b)
    with pytest.raises(wb.UnknownApproximantError):
        wb.to_physical_reference(b, 30.0, approximant="nope")
    from waveformx_b200._reference import REFERENCE_MODELS

    assert set(REFERENCE_MODELS) == {"TaylorF2", "IMRPhenomD", "IMRPhenomXAS", "IMRPhenomXHM"}


def test_modes_dispatch():
    """modes() of the reference: IMRPhenomXHM only (the aligned single-mode
    models raise UnsupportedError as the reference's); keywords checked
    before any device work; FrequencyModes indexing."""
    with pytest.raises(wb.UnsupportedError):
        wb.modes("IMRPhenomXAS", [20.0, 30.0], mass_1=30.0, mass_2=20.0)
    with pytest.raises(TypeError):
        wb.modes("IMRPhenomXHM", [20.0, 30.0], mass_1=30.0)
    with pytest.raises(TypeError):
        wb.modes("IMRPhenomXHM", [20.0, 30.0], mass_1=30.0, mass_2=20.0, chirp_mass=10.0)
    fm = wb.FrequencyModes(np.array([-2.0, -1.0, 1.0, 2.0]), {(2, 2): np.zeros(4), (2, -2): np.zeros(4)}, 0.3)
    f, m = fm
    assert fm[(2, 2)] is m[(2, 2)] and len(f) == 4
    hp, hc = fm.polarizations()
    assert hp.shape == (2,) and np.all(hp == 0) and np.all(hc == 0)


def test_offsets_and_per_frequency_checks():
    """The host checks of ragged offsets (the reference's rows check,
    src/waveformx/_api.py:292-305) and of the fused likelihood's data and
    weights sizes, on CPU tensors."""
    import torch

    from waveformx_b200.ops import check_per_frequency, offsets_problem

    assert offsets_problem(torch.tensor([0, 3, 3, 7]), 3, 7) is None
    assert offsets_problem(np.array([2, 3, 3, 7]), 3, 7) is None  # leading unused values are allowed
    assert "B + 1" in offsets_problem(torch.tensor([0, 3, 7]), 3, 7)
    assert "non-decreasing" in offsets_problem(torch.tensor([0, 5, 3, 7]), 3, 7)
    assert "non-decreasing" in offsets_problem(torch.tensor([0, 7, 0, 7]), 3, 7)
    assert "non-decreasing" in offsets_problem(torch.tensor([-1, 3, 3, 7]), 3, 7)
    assert "== 7" in offsets_problem(torch.tensor([0, 3, 3, 6]), 3, 7)
    assert "== 7" in offsets_problem(torch.tensor([0, 3, 3, 8]), 3, 7)
    shared, per_binary = torch.zeros(10), torch.zeros(40)
    assert check_per_frequency(shared, "data", 4, 10, False) == 0
    assert check_per_frequency(per_binary, "data", 4, 10, False) == 1
    assert check_per_frequency(shared, "weights", 4, 10, True) == 1
    with pytest.raises(ValueError, match="weights"):
        check_per_frequency(torch.zeros(39), "weights", 4, 10, False)
    with pytest.raises(ValueError, match="data"):
        check_per_frequency(torch.zeros(9), "data", 4, 10, True)
