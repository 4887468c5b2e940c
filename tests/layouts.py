"""The kernels' FP64 table layout (``waveformx_b200/csrc/tables.cuh``) mapped to
the oracle's dict and to the reference's flat tables (86 values for
IMRPhenomXAS, ``models/xas/core.py:68-89``; 75 for IMRPhenomD,
``models/phenomd/core.py:75-95``; 15 for TaylorF2,
``models/taylorf2/core.py:63-70``), so that tables computed on the GPU can
be compared with the golden ones."""

from __future__ import annotations

import numpy as np

from oracle import phenomd, taylorf2, xas


def xas_dict(tab: np.ndarray) -> dict:
    tab = np.asarray(tab, dtype=np.float64)
    b = len(tab)
    I = xas.INDEX
    ph = np.zeros((b, 3, 16))
    ph[:, 0, 1:14] = tab[:, 0:13]
    for j, k in enumerate([I[(0, 0)], I[(1, 0)], I[(0, 1)], I[(-1, 0)], I[(-2, 0)], I[(-3, 0)]]):
        ph[:, 1, k] = tab[:, 13 + j]
    for j, k in enumerate([I[(0, 0)], I[(1, 0)], I[(2 / 3, 0)], I[(-1, 0)], I[(-3, 0)]]):
        ph[:, 2, k] = tab[:, 19 + j]
    z = np.zeros(b)
    return dict(phase=ph, atan_a=np.stack([z, tab[:, 24], tab[:, 25]], -1),
                atan_w=np.stack([z, tab[:, 26], tab[:, 27]], -1), shift=tab[:, 28], amp_ins=tab[:, 29:39],
                amp_int_n=tab[:, 39], amp_int_d=tab[:, 40:45], amp_rd_n=tab[:, 45], amp_rd_gr=tab[:, 46],
                amp_rd_s=tab[:, 47], amp_rd_g=tab[:, 48], f_phase_in=tab[:, 49], f_phase_im=tab[:, 50],
                f_amp_in=tab[:, 51], f_amp_rd=tab[:, 52], f_cut=tab[:, 53], kp=tab[:, 54], kc=tab[:, 55],
                t0=tab[:, 56], anchor=tab[:, 57])


def phenomd_dict(tab: np.ndarray) -> dict:
    tab = np.asarray(tab, dtype=np.float64)
    b = len(tab)
    I = phenomd.INDEX
    ph = np.zeros((b, 3, 14))
    ins = [I[(0, 0)], I[(-1, 0)], I[(-2 / 3, 0)], I[(-1 / 3, 0)], I[(0, 1)], I[(1 / 3, 0)], I[(1 / 3, 1)],
           I[(2 / 3, 0)], I[(1, 0)], I[(4 / 3, 0)], I[(5 / 3, 0)], I[(2, 0)]]
    for j, k in enumerate(ins):
        ph[:, 0, k] = tab[:, j]
    for j, k in enumerate([I[(0, 0)], I[(1, 0)], I[(-3, 0)], I[(0, 1)]]):
        ph[:, 1, k] = tab[:, 12 + j]
    for j, k in enumerate([I[(0, 0)], I[(1, 0)], I[(-1, 0)], I[(3 / 4, 0)]]):
        ph[:, 2, k] = tab[:, 16 + j]
    return dict(phase=ph, atan_a=tab[:, 20], atan_w=tab[:, 21], atan_shift=tab[:, 22], amp_ins=tab[:, 23:33],
                amp_int=tab[:, 33:38], amp_int_s=tab[:, 38], amp_rd_n=tab[:, 39], amp_rd_gr=tab[:, 40],
                amp_rd_s=tab[:, 41], amp_rd_shift=tab[:, 42], f_phase_ins=tab[:, 43], f_phase_mrd=tab[:, 44],
                f_amp_ins=tab[:, 45], f_amp_mrd=tab[:, 46], kp=tab[:, 47], kc=tab[:, 48],
                t0=tab[:, 49], anchor=tab[:, 50])


def taylorf2_dict(tab: np.ndarray) -> dict:
    tab = np.asarray(tab, dtype=np.float64)
    return dict(phase=tab[:, 0:8], amp=tab[:, 9], kp=tab[:, 10], kc=tab[:, 11], t0=tab[:, 12], anchor=tab[:, 13])


def reference_flat(model: str, tab: np.ndarray) -> np.ndarray:
    """The reference's flat table of kernel tables ``(B, 72)``."""
    if model in ("xas", "IMRPhenomXAS"):
        return xas.flat(xas_dict(tab))
    if model in ("taylorf2", "TaylorF2"):
        return taylorf2.flat(taylorf2_dict(tab))
    return phenomd.flat(phenomd_dict(tab))


def relative_error(a: np.ndarray, b: np.ndarray) -> float:
    """The largest ``|a - b| / |b|`` (``|a|`` where ``b`` is zero)."""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    with np.errstate(invalid="ignore", divide="ignore"):
        r = np.where(b != 0, np.abs(a - b) / np.abs(b), np.abs(a))
    return float(np.nanmax(r))
