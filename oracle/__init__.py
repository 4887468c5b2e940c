"""The CPU oracle of the aligned-spin frequency-domain path: IMRPhenomXAS,
IMRPhenomD and TaylorF2 ``(hplus, hcross)`` in float64 NumPy, a
restatement of the reference's algorithm (``models/xas/core.py``,
``models/phenomd/core.py``, ``models/taylorf2/core.py`` and what they
call), vectorised over binaries.

TEST INFRASTRUCTURE ONLY. The tests, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` use it as the checker; the product
(``waveformx_b200``) never imports it. Its parity with the reference is
pinned by the golden vectors of ``tests/golden`` (written by the
reference's own code), which ``tests/test_oracle_golden.py`` checks.

Parameters are ``(B, 8)`` arrays with the columns ``mass_1, mass_2, chi_1,
chi_2, luminosity_distance, inclination, phi_ref, f_ref`` (solar masses,
Mpc, radians, Hz; ``f_ref = 0`` is the first frequency, or for TaylorF2
the reference at coalescence). The extension
``t_c`` (s) multiplies the strain by ``exp(-2 pi i f t_c)``.
"""

from .api import (  # noqa: F401
    MODELS,
    batch_loss,
    loss_gradient_fd,
    mismatch,
    phase_error,
    polarizations,
    psd,
    table,
)
