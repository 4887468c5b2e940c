"""Write the golden vectors of the reference-convention converters: the
reference's own ``to_mass_scaled_reference`` and ``to_physical_reference``
(``models/{taylorf2,phenomd,xas}/reference.py``, the functions that
``src/waveformx/_reference.py:59-80`` dispatches to; IMRPhenomXHM uses
IMRPhenomXAS's) run under the NumPy ``jax`` shim, one binary at a time, for
a seeded batch of binaries, half of them with ``f_ref = 0``.

Run from the repository root, in a container with the reference checkout:

    python tests/golden/make_golden_converters.py [--reference /path/to/waveformx]

The output, ``tests/golden/converters.npz``, is committed.
"""

from __future__ import annotations

import argparse
import importlib
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
from make_golden import draw_batch  # noqa: E402

MODULES = {"TaylorF2": "taylorf2", "IMRPhenomD": "phenomd", "IMRPhenomXAS": "xas"}
REFERENCE_MF, F_MIN, F_REF_OUT = 0.01, 20.0, 30.0


def main():
    parser = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    parser.add_argument("--reference", default=os.environ.get("WAVEFORMX_REFERENCE"),
                        required="WAVEFORMX_REFERENCE" not in os.environ,
                        help="the reference checkout's root (or the WAVEFORMX_REFERENCE environment variable)")
    parser.add_argument("--out", default=str(HERE))
    args = parser.parse_args()
    os.environ["WAVEFORMX_REFERENCE"] = args.reference
    import reference_loader

    ref = reference_loader.load()
    Binary = ref.binary.Binary
    params = draw_batch(np.random.default_rng(2026), 16)
    params[::2, 7] = 0.0  # f_ref = 0: the first frequency, or coalescence (TaylorF2)

    def binary(p):
        return Binary(np.float64(p[0]), np.float64(p[1]), np.array([0.0, 0.0, p[2]]), np.array([0.0, 0.0, p[3]]),
                      np.float64(p[4]), np.float64(p[5]), np.float64(p[6]), np.float64(p[7]))

    out = dict(params=params, reference_mf=REFERENCE_MF, f_min=F_MIN, f_ref_out=F_REF_OUT)
    for model, name in MODULES.items():
        module = importlib.import_module(f"waveformx.models.{name}.reference")
        scaled, physical = [], []
        for p in params:
            if name == "taylorf2":
                scaled.append(module.to_mass_scaled_reference(binary(p), REFERENCE_MF).phi_ref)
            else:
                scaled.append(module.to_mass_scaled_reference(binary(p), REFERENCE_MF, F_MIN).phi_ref)
            physical.append(module.to_physical_reference(binary(p), F_REF_OUT, REFERENCE_MF).phi_ref)
        out[f"{model}_scaled_phi_ref"] = np.asarray(scaled, np.float64)
        out[f"{model}_physical_phi_ref"] = np.asarray(physical, np.float64)
    np.savez_compressed(Path(args.out) / "converters.npz", **out)
    print({k: np.round(v[:3], 6) for k, v in out.items() if k.endswith("phi_ref")})


if __name__ == "__main__":
    main()
