"""Write the golden vectors of the aligned-spin frequency-domain path:
``(hplus, hcross)`` and the per-binary coefficient tables of IMRPhenomXAS
and IMRPhenomD, computed by the reference's own float64 code
(``models/xas/model.py:48-60``, ``models/phenomd/model.py:288-305``) run
under the NumPy ``jax`` shim of ``jaxshim/``.

Run from the repository root, in a container with the reference checkout:

    python tests/golden/make_golden.py [--reference /path/to/waveformx]

The output, ``tests/golden/*.npz``, is committed; the tests read only it.

Cases:

* ``xas_cases`` / ``phenomd_cases``: the hand-picked binaries of the
  reference's LAL comparisons (``tests/test_xas.py:28-39``,
  ``tests/test_phenomd.py:34-46``) on 256 geometric frequencies from their
  ``f_min`` to beyond the cutoff, plus the single-binary workload
  (36 + 29 Msun, chi = 0.3 / -0.1, 500 Mpc, inclination 0.7, phi_ref 1.2,
  f_ref 20 Hz, ``linspace(20, 1024, 4017)``);
* ``*_random``: 24 binaries drawn as the 4096-binary batch (seed 2024),
  on every 16th point of ``linspace(20, 1024, 4017)``;
* ``*_reference_mf``: four binaries with ``reference_mf = 0.01`` (f_ref = 0);
* ``*_unscaled``: two binaries with ``scaled_strain = False``;
* ``xas_nan``: a mass ratio of 2000 (NaN where LAL fails);
* ``qnm``: the (2,2) ring-down and damping frequencies of XAS at a few
  final spins, both the re-expanded form in ``1 - a`` and the direct fits.
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
XAS_CASES = [
    (30.0, 30.0, 0.0, 0.0, 400.0, 0.4, 0.0, 20.0, 20.0),
    (36.0, 29.0, 0.3, -0.4, 500.0, 1.0, 1.2, 20.0, 30.0),
    (60.0, 15.0, 0.8, 0.5, 1000.0, 2.5, 4.0, 15.0, 20.0),
    (80.0, 10.0, -0.7, 0.2, 2000.0, 2.0, 0.3, 10.0, 25.0),
    (1.6, 1.3, 0.05, 0.02, 40.0, 0.2, 2.0, 30.0, 40.0),
    (8.0, 1.4, 0.9, 0.0, 200.0, 0.3, 5.5, 20.0, 50.0),
    (150.0, 100.0, 0.95, 0.95, 3000.0, 0.7, 3.0, 10.0, 15.0),
    (25.0, 20.0, -0.9, -0.9, 300.0, 1.5, 0.7, 20.0, 20.0),
    (20.0, 45.0, 0.3, -0.4, 300.0, 2.9, 0.7, 20.0, 0.0),
    (50.0, 2.0, 0.995, 0.3, 300.0, 1.1, 1.7, 20.0, 25.0),
]
PHENOMD_CASES = XAS_CASES + [(90.0, 5.0, 1.0, 1.0, 300.0, 1.1, 1.7, 20.0, 0.0)]
SINGLE = (36.0, 29.0, 0.3, -0.1, 500.0, 0.7, 1.2, 20.0, 20.0)


def draw_batch(rng, n):
    """Binaries as the 4096-binary batch draws them: masses uniform 5-100
    sorted so that m1 >= m2, aligned spins uniform [-0.99, 0.99], distance
    uniform 100-5000 Mpc, cos(inclination) uniform [-1, 1], phi_ref uniform
    [0, 2 pi), f_ref = 20 Hz. Columns: m1, m2, chi1, chi2, D, iota, phi, f_ref."""
    m = rng.uniform(5.0, 100.0, size=(n, 2))
    m1, m2 = m.max(axis=1), m.min(axis=1)
    chi = rng.uniform(-0.99, 0.99, size=(n, 2))
    distance = rng.uniform(100.0, 5000.0, size=n)
    inclination = np.arccos(rng.uniform(-1.0, 1.0, size=n))
    phi = rng.uniform(0.0, 2.0 * np.pi, size=n)
    return np.stack([m1, m2, chi[:, 0], chi[:, 1], distance, inclination, phi, np.full(n, 20.0)], axis=1)


def case_grid(case, n, model):
    m1, m2, f_min = case[0], case[1], case[7]
    top = 0.33 / ((m1 + m2) * MTSUN_SI) * 1.05 if model == "xas" else 0.25 / ((m1 + m2) * MTSUN_SI)
    return np.geomspace(f_min, top, n)


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

    ref = reference_loader.load()
    Binary = ref.binary.Binary
    Options = ref.options.WaveformOptions

    def binary(p):
        return Binary(float(p[0]), float(p[1]), np.array([0.0, 0.0, p[2]]), np.array([0.0, 0.0, p[3]]),
                      float(p[4]), float(p[5]), float(p[6]), float(p[7]))

    models = {"xas": ref.xas_model, "phenomd": ref.phenomd_model}

    def run(model, params, grids, options):
        hp, hc, tables = [], [], []
        for p, f in zip(params, grids):
            a, b = models[model].polarizations(binary(p), np.asarray(f, dtype=np.float64), options)
            hp.append(np.asarray(a, np.complex128))
            hc.append(np.asarray(b, np.complex128))
            tables.append(table(model, p, f[0], options))
        return np.array(hp), np.array(hc), np.array(tables)

    def table(model, p, f_min, options):
        scale = ref.options.strain_scale(options)
        params = tuple(np.float64(x) for x in p)
        if model == "xas":
            params = ref.xas_model.with_reference(params, options.reference_mf)
            return np.asarray(ref.xas_core.table(params, np.float64(f_min), scale), np.float64)
        return np.asarray(ref.phenomd_core.table(params, np.float64(f_min), scale, options.reference_mf), np.float64)

    out = Path(args.out)
    default = Options()
    rng = np.random.default_rng(2024)
    random_params = draw_batch(rng, 24)
    shared = np.linspace(20.0, 1024.0, 4017)
    for model, cases in (("xas", XAS_CASES), ("phenomd", PHENOMD_CASES)):
        # the hand-picked cases, each on its own grid
        params = np.array([(c[0], c[1], c[2], c[3], c[4], c[5], c[6], c[8]) for c in cases])
        grids = np.array([case_grid(c, 256, model) for c in cases])
        hp, hc, tables = run(model, params, grids, default)
        # the single-binary workload
        sp = np.array([(SINGLE[0], SINGLE[1], SINGLE[2], SINGLE[3], SINGLE[4], SINGLE[5], SINGLE[6], SINGLE[8])])
        shp, shc, stab = run(model, sp, [shared], default)
        np.savez_compressed(out / f"{model}_cases.npz", params=params, frequencies=grids, hplus=hp, hcross=hc,
                            tables=tables, single_params=sp, single_frequencies=shared, single_hplus=shp[0],
                            single_hcross=shc[0], single_table=stab[0])
        # the random draw on a shared subsampled grid
        grid = shared[::16]
        hp, hc, tables = run(model, random_params, [grid] * len(random_params), default)
        np.savez_compressed(out / f"{model}_random.npz", params=random_params, frequencies=grid, hplus=hp,
                            hcross=hc, tables=tables, seed=2024)
        # the mass-scaled reference
        rp = params[:4].copy()
        rp[:, 7] = 0.0
        options = Options(reference_mf=0.01)
        rgrids = grids[:4]
        hp, hc, tables = run(model, rp, rgrids, options)
        np.savez_compressed(out / f"{model}_reference_mf.npz", params=rp, frequencies=rgrids, hplus=hp, hcross=hc,
                            tables=tables, reference_mf=0.01)
        # the strain itself
        options = Options(scaled_strain=False)
        hp, hc, tables = run(model, params[:2], grids[:2], options)
        np.savez_compressed(out / f"{model}_unscaled.npz", params=params[:2], frequencies=grids[:2], hplus=hp,
                            hcross=hc, tables=tables)
    # NaN where LAL fails (mass ratio 2000)
    bad = np.array([[2000.0, 1.0, 0.0, 0.0, 400.0, 0.4, 0.0, 20.0]])
    f = np.geomspace(20.0, 1024.0, 100)
    hp, hc, tables = run("xas", bad, [f], default)
    np.savez_compressed(out / "xas_nan.npz", params=bad, frequencies=f, hplus=hp, hcross=hc, tables=tables)
    # the QNM fits of XAS
    spins = np.array([-0.99, -0.5, 0.0, 0.5, 0.9, 0.99, 0.999])
    expanded = np.array([ref.xas_core.qnm_22(np.float64(a)) for a in spins])
    direct = np.array([(ref.qnm.fring22(a), ref.qnm.fdamp22(a)) for a in spins])
    np.savez_compressed(out / "qnm.npz", spins=spins, expanded=expanded, direct=direct)
    for path in sorted(out.glob("*.npz")):
        print(f"{path.name}: {path.stat().st_size / 1024:.0f} KiB")


if __name__ == "__main__":
    main()
