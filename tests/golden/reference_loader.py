"""Import the reference's aligned-spin frequency-domain modules (IMRPhenomXAS,
IMRPhenomD, TaylorF2, IMRPhenomXHM and what they use) from a read-only checkout, under the NumPy
``jax`` shim of ``jaxshim/``, without running the package's ``__init__``
(which imports every model and JAX itself).

Only ``make_golden.py``, ``make_golden_taylorf2.py`` and ``make_golden_xhm.py`` use this, in a container that has the reference
checkout; the committed fixtures it writes are what the tests read.
"""

from __future__ import annotations

import importlib
import os
import sys
import types
from pathlib import Path

HERE = Path(__file__).resolve().parent


def source() -> Path:
    """The reference checkout's package directory, from the
    ``WAVEFORMX_REFERENCE`` environment variable (the checkout's root; no
    default: the scripts' ``--reference`` sets it)."""
    root = os.environ.get("WAVEFORMX_REFERENCE")
    if not root:
        raise RuntimeError("set WAVEFORMX_REFERENCE (or pass --reference) to the reference checkout's root")
    return Path(root) / "src" / "waveformx"

_PACKAGES = ("waveformx", "waveformx.models", "waveformx.models.xpnr", "waveformx.models.xas",
             "waveformx.models.phenomd", "waveformx.models.taylorf2", "waveformx.models.xhm",
             "waveformx.models.xpnr.hm", "waveformx.models.xpnr._generated")


def load():
    """The modules of the reference, as a namespace: ``xas_core``,
    ``xas_model``, ``phenomd_core``, ``phenomd_model``, ``phenomd_fits``,
    ``taylorf2_core``, ``taylorf2_model``, ``options``, ``binary``, ``qnm``,
    ``pn``, ``xhm_core``, ``xhm_model``, ``xhm_reference``."""
    source_dir = source()
    if not source_dir.is_dir():
        raise FileNotFoundError(f"the reference checkout is not at {source_dir}")
    shim = str(HERE / "jaxshim")
    if shim not in sys.path:
        sys.path.insert(0, shim)
    import jax  # noqa: F401  (the shim)

    assert getattr(jax, "__version__", "") == "0.0-numpy-shim", "a real JAX shadows the shim"
    for name in _PACKAGES:
        if name in sys.modules:
            continue
        package = types.ModuleType(name)
        package.__path__ = [str(source_dir.joinpath(*name.split(".")[1:]))]
        sys.modules[name] = package
    imp = importlib.import_module
    return types.SimpleNamespace(
        xas_core=imp("waveformx.models.xas.core"),
        xas_model=imp("waveformx.models.xas.model"),
        phenomd_core=imp("waveformx.models.phenomd.core"),
        phenomd_model=imp("waveformx.models.phenomd.model"),
        phenomd_fits=imp("waveformx.models.phenomd.fits"),
        options=imp("waveformx._options"),
        binary=imp("waveformx._binary"),
        qnm=imp("waveformx.models.xpnr._generated.qnm"),
        pn=imp("waveformx.models.taylorf2.pn"),
        taylorf2_core=imp("waveformx.models.taylorf2.core"),
        taylorf2_model=imp("waveformx.models.taylorf2.model"),
        xhm_core=imp("waveformx.models.xhm.core"),
        xhm_model=imp("waveformx.models.xhm.model"),
        xhm_reference=imp("waveformx.models.xhm.reference"),
    )
