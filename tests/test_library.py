"""The C-ABI library on a machine without a GPU: it is built for sm_100a,
loads, and exports every entry point ``include/waveformx_b200.h`` declares,
with the binding's prototypes; host-only entries answer. No kernel runs."""

from __future__ import annotations

import re
import subprocess
import sys

import pytest

from conftest import ROOT

HEADER = ROOT / "include" / "waveformx_b200.h"


def declared():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(wfx_[a-z_0-9]+)\s*\(", text)))


def test_header_declares_the_binding():
    from waveformx_b200 import _lib

    assert declared() == sorted(_lib.EXPORTS)


def test_library_loads_and_exports_every_symbol():
    from waveformx_b200 import _build, _lib

    if _build.stale():
        pytest.skip("the library is not built (python -m waveformx_b200._build)")
    lib = _lib.library()
    for name in declared():
        assert hasattr(lib, name), name
    nm = subprocess.run(["nm", "-D", "--defined-only", str(_build.LIBRARY)], capture_output=True, text=True)
    if nm.returncode == 0:
        exported = set(re.findall(r"\bT (wfx_\w+)", nm.stdout))
        assert set(declared()) <= exported
    assert lib.wfx_version() == 100
    assert b"invalid" in lib.wfx_status_string(-1)
    assert b"static scratch" in lib.wfx_status_string(_lib.ESCRATCH)
    assert lib.wfx_workspace_bytes(_lib.OP_FUSED, _lib.XAS, _lib.FP32, 1024, 4017, 0) > 0
    assert lib.wfx_workspace_bytes(_lib.OP_FUSED, _lib.XAS, _lib.FP64, 1024, 4017, 0) == 0
    assert lib.wfx_workspace_bytes(_lib.OP_POLARIZATIONS, _lib.XAS, _lib.FP32, 16, 1000, 1) > 0
    assert lib.wfx_workspace_bytes(_lib.OP_POLARIZATIONS, _lib.XAS, _lib.FP32, 16, 1000, 0) == 0


def test_library_is_sm100a():
    """The fat binary holds sm_100a code (cuobjdump is not used: the ELF's
    embedded-architecture note is read from the build flags)."""
    from waveformx_b200 import _build

    assert "arch=compute_100a,code=sm_100a" in " ".join(_build.NVCC_FLAGS)
    assert set(_build.UNITS) == {"kernels.cu", "setup.cu", "match.cu"}


def test_import_does_not_import_torch():
    code = "import sys, waveformx_b200; assert 'torch' not in sys.modules"
    subprocess.run([sys.executable, "-c", code], check=True, cwd=str(ROOT))


def test_entries_fail_loudly_without_a_device():
    """Without CUDA the product raises KernelError; it never falls back to
    a CPU path."""
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    import waveformx_b200 as wb

    with pytest.raises(wb.KernelError):
        wb.batch_polarizations("IMRPhenomXAS", [20.0, 30.0], [[36.0, 29.0] + [0.0] * 6 + [500.0, 0.7, 1.2, 20.0]])
    f = wb.polarizations_function("IMRPhenomXAS")
    with pytest.raises(wb.KernelError):
        f(wb.Binary(36.0, 29.0, (0, 0, 0), (0, 0, 0)), torch.tensor([20.0, 30.0]))
