"""Write the golden vectors of IMRPhenomXHM (the aligned-spin model with
higher modes): the per-binary coefficient tables, the modes
``h_{l,-m}`` of ``(2,2), (2,1), (3,3), (3,2), (4,4)`` and ``(hplus,
hcross)``, computed by the reference's own float64 code
(``models/xhm/core.py:388-397`` for the table, ``models/xhm/model.py:30-42``
for the modes and polarizations) run under the NumPy ``jax`` shim of
``jaxshim/`` (whose ``jvp`` is forward mode on dual numbers, for the two
exact derivatives of the set-up, ``models/xhm/reference.py:72-74``).

Run from the repository root, in a container with the reference checkout:

    python tests/golden/make_golden_xhm.py [--reference /path/to/waveformx]

The output, ``tests/golden/xhm_*.npz``, is committed; the tests read only it.

Cases:

* ``xhm_cases``: the hand-picked binaries of ``make_golden.py`` (the
  reference's LAL comparisons, ``tests/test_xas.py:28-39``) and a mass
  ratio of 100 with a negative primary spin (the (3,2) phase boundary moved,
  ``models/xhm/reference.py:412``), each on 256 geometric frequencies from
  its ``f_min`` to ``0.45 / M`` (past every mode's ringdown);
* ``xhm_random``: 24 binaries drawn as the 4096-binary batch (seed 2025) on
  every 16th point of ``linspace(20, 1024, 4017)``;
* ``xhm_reference_mf``: four binaries with ``reference_mf = 0.01``;
* ``xhm_unscaled``: two binaries with ``scaled_strain = False``.
"""

from __future__ import annotations

import argparse
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
from make_golden import MTSUN_SI, XAS_CASES, draw_batch  # noqa: E402

# mass_1, mass_2, chi_1, chi_2, distance, inclination, phi_ref, f_min, f_ref
XHM_CASES = XAS_CASES + [(100.0, 1.0, -0.5, 0.2, 300.0, 0.9, 0.4, 20.0, 20.0)]


def case_grid(case, n):
    m1, m2, f_min = case[0], case[1], case[7]
    return np.geomspace(f_min, 0.45 / ((m1 + m2) * MTSUN_SI), n)


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
    Options = ref.options.WaveformOptions
    core, model = ref.xhm_core, ref.xhm_model

    def binary(p):
        return Binary(float(p[0]), float(p[1]), np.array([0.0, 0.0, p[2]]), np.array([0.0, 0.0, p[3]]),
                      float(p[4]), float(p[5]), float(p[6]), float(p[7]))

    def run(params, grids, options):
        out = dict(hplus=[], hcross=[], modes=[], tables=[])
        scale = ref.options.strain_scale(options)
        for p, f in zip(params, grids):
            f = np.asarray(f, dtype=np.float64)
            modes, (hp, hc) = model.modes_and_polarizations(binary(p), f, options)
            out["hplus"].append(np.asarray(hp, np.complex128))
            out["hcross"].append(np.asarray(hc, np.complex128))
            out["modes"].append(np.stack([np.asarray(modes[m], np.complex128) for m in core.MODES]))
            aligned = ref.xas_model.with_reference(tuple(np.float64(x) for x in p), options.reference_mf)
            out["tables"].append(np.asarray(core.table(aligned, np.float64(f[0]), scale), np.float64))
        return {k: np.array(v) for k, v in out.items()}

    out = Path(args.out)
    default = Options()
    modes = np.array(core.MODES)
    params = np.array([(c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[8]) for c in XHM_CASES])
    grids = np.array([case_grid(c, 256) for c in XHM_CASES])
    np.savez_compressed(out / "xhm_cases.npz", params=params, frequencies=grids, mode_list=modes,
                        **run(params, grids, default))
    rng = np.random.default_rng(2025)
    random_params = draw_batch(rng, 24)
    grid = np.linspace(20.0, 1024.0, 4017)[::16]
    np.savez_compressed(out / "xhm_random.npz", params=random_params, frequencies=grid, mode_list=modes, seed=2025,
                        **run(random_params, [grid] * len(random_params), default))
    rp = params[:4].copy()
    rp[:, 7] = 0.0
    np.savez_compressed(out / "xhm_reference_mf.npz", params=rp, frequencies=grids[:4], mode_list=modes,
                        reference_mf=0.01, **run(rp, grids[:4], Options(reference_mf=0.01)))
    np.savez_compressed(out / "xhm_unscaled.npz", params=params[:2], frequencies=grids[:2], mode_list=modes,
                        **run(params[:2], grids[:2], Options(scaled_strain=False)))
    for path in sorted(out.glob("xhm_*.npz")):
        print(f"{path.name}: {path.stat().st_size / 1024:.0f} KiB")


if __name__ == "__main__":
    main()
