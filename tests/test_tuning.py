"""The ragged forward's tuning table on the host (no GPU needed): the JSON
record and the library's process-wide table."""

from __future__ import annotations

import pytest

from waveformx_b200 import tuning


def test_size_class():
    assert tuning.size_class(16384, 272782499) == "28,14"
    assert tuning.size_class(1, 1) == "0,0"


def test_json_round_trip(tmp_path):
    path = tmp_path / "tuning.json"
    tuning.save_entry("NVIDIA B200", "IMRPhenomXAS", "28,14", (2046, 8), path)
    tuning.save_entry("NVIDIA B200", "IMRPhenomD", "20,10", (510, 4), path)
    tuning.save_entry("other", "IMRPhenomXAS", "28,14", (4094, 2), path)
    data = tuning._read(path)
    assert data["NVIDIA B200"]["IMRPhenomXAS"]["28,14"] == [2046, 8]
    assert data["NVIDIA B200"]["IMRPhenomD"]["20,10"] == [510, 4]
    assert data["other"]["IMRPhenomXAS"]["28,14"] == [4094, 2]


def test_library_table(tmp_path):
    from waveformx_b200 import _build

    if _build.stale():
        pytest.skip("the library is not built")
    path = tmp_path / "tuning.json"
    tuning.save_entry("dev", "IMRPhenomXAS", tuning.size_class(3000, 5_000_000), (2046, 16), path)
    assert tuning.load("dev", path) == 1
    assert tuning.lookup("IMRPhenomXAS", 3000, 5_000_000) == (2046, 16, True)
    # the same size class
    assert tuning.lookup("IMRPhenomXAS", 2048, 4_194_304) == (2046, 16, True)
    untuned = tuning.lookup("IMRPhenomD", 3000, 5_000_000)
    assert untuned[2] is False and untuned[0] >= 510
    from waveformx_b200 import KernelError

    with pytest.raises(KernelError):
        tuning.install("IMRPhenomXAS", 10, 10, 100, 8)  # item length below the shortest
