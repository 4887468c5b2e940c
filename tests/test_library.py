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
    assert set(_build.UNITS) == {"kernels.cu", "setup.cu", "match.cu", "xhm.cu", "pipeline.cu"}


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


def test_match_entries_check_their_time_mode():
    """The refinement's time modes (0 none, 1 from the grid, 2 from given
    times) and the grid-time entry's lengths are checked before any launch:
    WFX_EINVAL for a missing grid, missing times, an unknown mode or an
    unsupported length; a valid call reaches the device (here: none) and
    returns its error (host code that ran a device-only helper would end
    the process instead). The valid calls are made only where no CUDA
    device is present: their buffers are host memory."""
    import ctypes

    from waveformx_b200 import _lib

    torch = pytest.importorskip("torch")
    device_present = torch.cuda.is_available()

    lib = _lib.library()
    buf = (ctypes.c_double * 64)()
    p = ctypes.addressof(buf)
    einval = -1

    def refine(zgrid, time, t):
        return lib.wfx_match_refine(_lib.FP32, p, zgrid, 4, 10, 16, p, 0.25, p, time, 1, 3, p, t, None)

    assert refine(None, 1, p) == einval
    assert refine(None, 2, None) == einval
    assert refine(p, 3, p) == einval
    assert refine(None, -1, p) == einval
    assert lib.wfx_match_grid_time(p, 4, 10, 4096, 0.25, None, None) == einval
    from waveformx_b200 import ops

    sizes = ((10, 2048), (10, 3072), (1969, 8192), (4017, 16384), (3000, 8192), (5000, 16384),
             (9000, 16384), (9000, 8192), (20000, 32768), (2049, 6144), (1000, 4096), (4096, 4096))
    for n, n_fft in sizes:
        if not ops.grid_time_supported(n, n_fft):
            assert lib.wfx_match_grid_time(p, 4, n, n_fft, 0.25, p, None) == einval, (n, n_fft)
    if device_present:
        return
    for zgrid, time in ((None, 0), (p, 1), (None, 2)):
        assert refine(zgrid, time, p) not in (0, einval)
    for n, n_fft in sizes:
        if ops.grid_time_supported(n, n_fft):
            assert lib.wfx_match_grid_time(p, 4, n, n_fft, 0.25, p, None) not in (0, einval), (n, n_fft)


def test_batch_and_jvp_entries_check_their_arguments():
    """wfx_pipeline_likelihood_run and wfx_xhm_setup_jvp refuse bad arguments
    before any launch: WFX_EINVAL for a missing buffer, IMRPhenomXHM in the
    likelihood, a group over per-binary f_min or a misaligned FP32 table;
    WFX_EWORKSPACE for a workspace smaller than two halves of
    wfx_workspace_bytes (the buffers are host memory: nothing reaches a
    device)."""
    import ctypes

    from waveformx_b200 import _lib

    lib = _lib.library()
    buf = (ctypes.c_double * 4096)()
    p = ctypes.addressof(buf)
    B, n, K = 4, 101, 3
    half = lib.wfx_workspace_bytes(_lib.OP_FUSED, _lib.XAS, _lib.FP32, B, n, 0)
    assert half > 0

    def run(model=_lib.XAS, pipe=p, group=1, f_stride=0, workspace=p, ws_bytes=None, loss=p):
        ws_bytes = 2 * half if ws_bytes is None else ws_bytes
        return lib.wfx_pipeline_likelihood_run(pipe, model, K, p, B, p, f_stride, 1e21, float("nan"), p, p, p, p,
                                               None, n, None, p, 0, p, 0, 1.0, 0.0, -0.5, loss, p, group,
                                               workspace, ws_bytes, None)

    assert run(pipe=None) == _lib.EINVAL
    assert run(model=_lib.XHM) == _lib.EINVAL
    assert run(group=2, f_stride=1) == _lib.EINVAL
    assert run(loss=None) == _lib.EINVAL
    assert run(ws_bytes=2 * half - 1) == _lib.EWORKSPACE
    assert run(workspace=None) == _lib.EWORKSPACE

    def jvp(dtable=p, table32=None, batch=B):
        return lib.wfx_xhm_setup_jvp(p, batch, p, 0, 1e21, float("nan"), None, table32, dtable, None, None)

    assert jvp(dtable=None) == _lib.EINVAL
    assert jvp(batch=0) == _lib.EINVAL
    assert jvp(table32=p + 4) == _lib.EINVAL


def test_grid_vjp_checks_its_arguments():
    """wfx_grid_vjp, the derivative with respect to the grid of every model
    (IMRPhenomXHM included), refuses before any CUDA call: WFX_EINVAL for a
    missing buffer, a non-positive size or an unknown model code (the
    buffers are host memory: nothing reaches a device)."""
    import ctypes

    from waveformx_b200 import _lib

    lib = _lib.library()
    buf = (ctypes.c_double * 64)()
    p = ctypes.addressof(buf)

    def run(model, table=p, grad=p, batch=2, n=8):
        return lib.wfx_grid_vjp(model, table, p, None, batch, n, None, p, p, grad, None)

    for model in (_lib.XAS, _lib.PHENOMD, _lib.TAYLORF2, _lib.XHM):
        assert run(model, table=None) == _lib.EINVAL
        assert run(model, grad=None) == _lib.EINVAL
        assert run(model, batch=0) == _lib.EINVAL
        assert run(model, n=0) == _lib.EINVAL
    assert run(_lib.XHM + 1) == _lib.EINVAL
    assert run(-1) == _lib.EINVAL


def test_reverse_pass_items_follow_the_batch():
    """The reverse pass's work items (one 64-float row of partial sums each in
    the workspace): a shared grid splits into tiles of at most 2046, 1022 or
    510 frequencies, the longest that still gives 8192 items (1024 x 4017:
    8 tiles a binary; 65536 x 8192: 5), so the workspace of a small batch
    holds more items per binary than a large one's."""
    from waveformx_b200 import _lib

    lib = _lib.library()

    def items(batch, n):
        return lib.wfx_workspace_bytes(_lib.OP_FUSED, _lib.XAS, _lib.FP32, batch, n, 0) // (64 * 4)

    assert 8192 <= items(1024, 4017) < 8192 + 64
    assert 5 * 65536 <= items(65536, 8192) < 5 * 65536 + 64
    assert 2 * 4096 <= items(4096, 4017) < 2 * 4096 + 64
    assert 4 * 2048 <= items(2048, 4017) < 4 * 2048 + 64
    assert items(16, 4017) >= 8 * 16
