"""Autotuning of the FP32 ragged forward.

The persistent kernel of a ragged batch takes (binary, tile) work items; the
tile length and the number of resident blocks per SM trade load balance
against per-item overhead, and the best pair depends on the batch. The
library times the candidates on a real problem (``wfx_autotune_ragged``)
and keeps the winner per device, model and size class (log2 of the number
of frequencies and of binaries) in a process-wide table; this module runs
it from PyTorch tensors and persists the table as JSON between processes
(``WAVEFORMX_B200_TUNING``, default ``~/.cache/waveformx_b200/tuning.json``),
keyed by the device name.
"""

from __future__ import annotations

import ctypes
import json
import os
import threading
from pathlib import Path
from typing import Optional

from . import _lib

__all__ = ["autotune_ragged", "install", "load", "lookup", "save_entry", "default_path", "size_class"]

_lock = threading.Lock()


def default_path() -> Path:
    env = os.environ.get("WAVEFORMX_B200_TUNING")
    return Path(env) if env else Path.home() / ".cache" / "waveformx_b200" / "tuning.json"


def size_class(batch: int, n: int) -> str:
    """The key of a problem's size class: ``"log2 n,log2 B"``."""
    return f"{max(int(n), 1).bit_length() - 1},{max(int(batch), 1).bit_length() - 1}"


def _model(approximant: str) -> int:
    from .ops import model_code

    return model_code(approximant)


def lookup(approximant: str, batch: int, n: int) -> tuple[int, int, bool]:
    """``(item length, blocks per SM, tuned)`` that the library uses for a
    ragged problem of ``batch`` binaries and ``n`` frequencies on the current
    device."""
    config = (ctypes.c_int64 * 2)()
    tuned = _lib.library().wfx_tuning(_model(approximant), int(batch), int(n), config, 0)
    if tuned < 0:
        _lib.check("wfx_tuning", tuned)
    return int(config[0]), int(config[1]), bool(tuned)


def install(approximant: str, batch: int, n: int, tile_len: int, blocks_per_sm: int) -> None:
    """Install a tuning for the size class of (batch, n) on the current device."""
    config = (ctypes.c_int64 * 2)(int(tile_len), int(blocks_per_sm))
    rc = _lib.library().wfx_tuning(_model(approximant), int(batch), int(n), config, 1)
    if rc != 1:
        _lib.check("wfx_tuning", rc if rc < 0 else -1)


def _read(path: Path) -> dict:
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return {}


def save_entry(device_name: str, approximant: str, key: str, config, path: Optional[Path] = None) -> None:
    """Record one tuning in the JSON file (merged with what is there)."""
    path = Path(path) if path is not None else default_path()
    with _lock:
        data = _read(path)
        data.setdefault(device_name, {}).setdefault(approximant, {})[key] = [int(config[0]), int(config[1])]
        path.parent.mkdir(parents=True, exist_ok=True)
        tmp = path.with_suffix(".tmp")
        tmp.write_text(json.dumps(data, indent=1, sort_keys=True))
        os.replace(tmp, path)


def load(device_name: str, path: Optional[Path] = None) -> int:
    """Install every tuning recorded for ``device_name`` (on the current
    device); returns how many."""
    path = Path(path) if path is not None else default_path()
    count = 0
    for approximant, entries in _read(path).get(device_name, {}).items():
        for key, (tile_len, blocks_per_sm) in entries.items():
            log_n, log_b = (int(v) for v in key.split(","))
            install(approximant, 1 << log_b, 1 << log_n, tile_len, blocks_per_sm)
            count += 1
    return count


def autotune_ragged(approximant: str, table, freqs, offsets, t_c=None, *, save: bool = True,
                    path: Optional[Path] = None) -> tuple[int, int]:
    """Time the candidate tilings of the ragged forward on this problem
    (FP32 ``table`` from the set-up, flat ``freqs``, ``offsets``), install
    the fastest for its size class and (``save``) record it in the JSON
    file. Synchronises the device; not for use inside a stream capture."""
    import torch

    from .ops import _ptr, _stream, workspace

    model = _model(approximant)
    batch, n = table.shape[0], freqs.numel()
    hp = torch.empty(n, dtype=torch.complex64, device=table.device)
    hc = torch.empty_like(hp)
    ws = workspace(_lib.OP_POLARIZATIONS, model, _lib.FP32, batch, n, True, table.device)
    config = (ctypes.c_int64 * 2)()
    _lib.check("wfx_autotune_ragged", _lib.library().wfx_autotune_ragged(
        model, _ptr(table), _ptr(freqs), _ptr(offsets), batch, n, _ptr(t_c), _ptr(hp), _ptr(hc), _ptr(ws),
        ws.numel(), _stream(table.device), config))
    result = (int(config[0]), int(config[1]))
    if save:
        save_entry(torch.cuda.get_device_name(table.device), approximant, size_class(batch, n), result, path)
    return result
