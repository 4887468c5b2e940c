"""Write the golden vectors of TaylorF2: ``(hplus, hcross)`` and the
per-binary coefficient tables, computed by the reference's own float64 code
(``models/taylorf2/model.py:24-35``, ``models/taylorf2/core.py:107-165``)
run under the NumPy ``jax`` shim of ``jaxshim/``.

Run from the repository root, in a container with the reference checkout:

    python tests/golden/make_golden_taylorf2.py [--reference /path/to/waveformx]

The output, ``tests/golden/taylorf2_*.npz``, is committed; the tests read
only it.

Cases:

* ``taylorf2_cases``: the hand-picked binaries of the reference's LAL
  comparison (``tests/test_taylorf2.py:25-34``; ``f_ref = 0`` is the
  reference at coalescence) on 256 geometric frequencies from their
  ``f_min`` to 1.5 times the Schwarzschild ISCO frequency
  (``tests/test_taylorf2.py:46-51``), plus the single-binary workload
  (36 + 29 Msun, chi = 0.3 / -0.1, 500 Mpc, inclination 0.7, phi_ref 1.2,
  f_ref 20 Hz, ``linspace(20, 1024, 4017)``) and a binary neutron star on
  a 1/256 Hz grid from 20 Hz (``tests/test_taylorf2.py:97-109``, every
  64th point);
* ``taylorf2_random``: 24 binaries drawn as the 4096-binary batch
  (seed 2024), on every 16th point of ``linspace(20, 1024, 4017)``;
* ``taylorf2_reference_mf``: four binaries with ``reference_mf = 0.01``
  (f_ref = 0), and one with f_ref = 20 Hz that the reference refuses (NaN);
* ``taylorf2_unscaled``: two binaries with ``scaled_strain = False``.
"""

from __future__ import annotations

import argparse
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
MTSUN_SI = 4.925490947641267e-06

# mass_1, mass_2, chi_1, chi_2, distance, inclination, phi_ref, f_min, f_ref
CASES = [
    (30.0, 30.0, 0.0, 0.0, 400.0, 0.4, 0.0, 20.0, 20.0),
    (36.0, 29.0, 0.3, -0.4, 500.0, 1.0, 1.2, 20.0, 0.0),
    (60.0, 15.0, 0.8, 0.5, 1000.0, 2.5, 4.0, 15.0, 20.0),
    (1.6, 1.3, 0.05, 0.02, 40.0, 0.2, 2.0, 20.0, 40.0),
    (8.0, 1.4, 0.9, 0.0, 200.0, 0.3, 5.5, 20.0, 0.0),
    (25.0, 20.0, -0.9, -0.9, 300.0, 1.5, 0.7, 20.0, 20.0),
    (20.0, 45.0, 0.3, -0.4, 300.0, 2.9, 0.7, 20.0, 0.0),
    (50.0, 2.0, 0.995, 0.3, 300.0, 1.1, 1.7, 10.0, 25.0),
]
SINGLE = (36.0, 29.0, 0.3, -0.1, 500.0, 0.7, 1.2, 20.0, 20.0)
BNS = (1.42, 1.27, 0.05, -0.03, 100.0, 0.5, 1.0, 20.0, 30.0)


def case_grid(case, n):
    m1, m2, f_min = case[0], case[1], case[7]
    return np.geomspace(f_min, 1.5 / (6.0 ** 1.5 * np.pi * (m1 + m2) * MTSUN_SI), n)


def main():
    parser = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    parser.add_argument("--reference", default=os.environ.get("WAVEFORMX_REFERENCE"),
                        required="WAVEFORMX_REFERENCE" not in os.environ,
                        help="the reference checkout's root (or the WAVEFORMX_REFERENCE environment variable)")
    parser.add_argument("--out", default=str(HERE))
    args = parser.parse_args()
    os.environ["WAVEFORMX_REFERENCE"] = args.reference
    sys.path.insert(0, str(HERE))
    import reference_loader
    from make_golden import draw_batch

    ref = reference_loader.load()
    Binary = ref.binary.Binary
    Options = ref.options.WaveformOptions

    def binary(p):
        return Binary(float(p[0]), float(p[1]), np.array([0.0, 0.0, p[2]]), np.array([0.0, 0.0, p[3]]),
                      float(p[4]), float(p[5]), float(p[6]), float(p[7]))

    def run(params, grids, options):
        hp, hc, tables = [], [], []
        for p, f in zip(params, grids):
            a, b = ref.taylorf2_model.polarizations(binary(p), np.asarray(f, dtype=np.float64), options)
            hp.append(np.asarray(a, np.complex128))
            hc.append(np.asarray(b, np.complex128))
            scale = ref.options.strain_scale(options)
            tables.append(np.asarray(ref.taylorf2_core.table(tuple(np.float64(x) for x in p), scale,
                                                             options.reference_mf), np.float64))
        return np.array(hp), np.array(hc), np.array(tables)

    out = Path(args.out)
    default = Options()
    params = np.array([(c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[8]) for c in CASES])
    grids = np.array([case_grid(c, 256) for c in CASES])
    hp, hc, tables = run(params, grids, default)
    shared = np.linspace(20.0, 1024.0, 4017)
    sp = np.array([(SINGLE[0], SINGLE[1], SINGLE[2], SINGLE[3], SINGLE[4], SINGLE[5], SINGLE[6], SINGLE[8])])
    shp, shc, stab = run(sp, [shared], default)
    bp = np.array([(BNS[0], BNS[1], BNS[2], BNS[3], BNS[4], BNS[5], BNS[6], BNS[8])])
    bns_grid = (20.0 + np.arange((2048 - 20) * 256) / 256.0)[::64]
    bhp, bhc, btab = run(bp, [bns_grid], default)
    np.savez_compressed(out / "taylorf2_cases.npz", params=params, frequencies=grids, hplus=hp, hcross=hc,
                        tables=tables, single_params=sp, single_frequencies=shared, single_hplus=shp[0],
                        single_hcross=shc[0], single_table=stab[0], bns_params=bp, bns_frequencies=bns_grid,
                        bns_hplus=bhp[0], bns_hcross=bhc[0], bns_table=btab[0])
    rng = np.random.default_rng(2024)
    random_params = draw_batch(rng, 24)
    grid = shared[::16]
    hp, hc, tables = run(random_params, [grid] * len(random_params), default)
    np.savez_compressed(out / "taylorf2_random.npz", params=random_params, frequencies=grid, hplus=hp, hcross=hc,
                        tables=tables, seed=2024)
    rp = params[:5].copy()
    rp[:4, 7] = 0.0
    rp[4, 7] = 20.0  # refused: f_ref must be zero with reference_mf
    options = Options(reference_mf=0.01)
    hp, hc, tables = run(rp, grids[:5], options)
    np.savez_compressed(out / "taylorf2_reference_mf.npz", params=rp, frequencies=grids[:5], hplus=hp, hcross=hc,
                        tables=tables, reference_mf=0.01)
    options = Options(scaled_strain=False)
    hp, hc, tables = run(params[:2], grids[:2], options)
    np.savez_compressed(out / "taylorf2_unscaled.npz", params=params[:2], frequencies=grids[:2], hplus=hp,
                        hcross=hc, tables=tables)
    for path in sorted(out.glob("taylorf2_*.npz")):
        print(f"{path.name}: {path.stat().st_size / 1024:.0f} KiB")


if __name__ == "__main__":
    main()
