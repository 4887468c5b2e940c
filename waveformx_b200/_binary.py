"""The parameters of a binary: the reference's ``Binary`` namedtuple and
``(n, 12)`` parameter table (``src/waveformx/_binary.py:18-183``), with
vectorised forms of its common checks for whole tables."""

from __future__ import annotations

from typing import Any, Mapping, NamedTuple

import numpy as np

from .exceptions import InvalidParameterError

__all__ = ["Binary", "BINARY_NAMES", "COLUMNS", "parameter_table", "check_binary", "table_errors", "aligned_table"]


class Binary(NamedTuple):
    """The parameters of ``SimInspiralChooseFDWaveform`` (masses in solar
    masses, distance in Mpc), as the reference's ``Binary``. Fields may be
    numbers, arrays or torch tensors, with a leading batch axis (``spin_1``,
    ``spin_2`` then ``(n, 3)``)."""

    mass_1: Any
    mass_2: Any
    spin_1: Any
    spin_2: Any
    luminosity_distance: Any = 1.0
    inclination: Any = 0.0
    phi_ref: Any = 0.0
    f_ref: Any = 0.0


BINARY_NAMES = Binary._fields

#: The columns of a parameter table.
COLUMNS = ("mass_1", "mass_2", "spin_1x", "spin_1y", "spin_1z", "spin_2x", "spin_2y", "spin_2z",
           "luminosity_distance", "inclination", "phi_ref", "f_ref")


def parameter_table(parameters: Any) -> np.ndarray:
    """An ``(n, 12)`` float64 table with the columns of :data:`COLUMNS`, from
    a mapping of arrays (``spin_1``/``spin_2`` as ``(n, 3)`` or the columns
    ``spin_1x`` ...; missing optional parameters take their defaults), a
    structured array or a ``DataFrame``, or an ``(n, 12)`` array."""
    names = None
    if isinstance(parameters, Mapping):
        names = set(parameters.keys())
    elif getattr(getattr(parameters, "dtype", None), "names", None):
        names = set(parameters.dtype.names)
    elif hasattr(parameters, "columns"):
        names = set(parameters.columns)
    if names is not None:
        if not names:
            raise TypeError("parameters is empty")
        n = len(np.atleast_1d(np.asarray(parameters[next(iter(names))])))
        unknown = names - set(COLUMNS) - set(BINARY_NAMES)
        if unknown:
            raise TypeError(f"unknown parameters {sorted(unknown)}: the columns are {', '.join(COLUMNS)}")
        columns = []
        for column in COLUMNS:
            if column in names:
                values = np.asarray(parameters[column], dtype=float)
            elif column[:-1] in ("spin_1", "spin_2") and column[:-1] in names:
                values = np.asarray(parameters[column[:-1]], dtype=float).reshape(n, 3)[:, "xyz".index(column[-1])]
            elif column in ("mass_1", "mass_2"):
                raise TypeError(f"parameters must contain {column!r}")
            else:
                values = np.full(n, Binary._field_defaults.get(column, 0.0), dtype=float)
            columns.append(np.broadcast_to(values, (n,)))
        return np.stack(columns, axis=1)
    table = np.asarray(parameters, dtype=float)
    if table.ndim != 2 or table.shape[1] != len(COLUMNS):
        raise ValueError(f"parameters must have {len(COLUMNS)} columns ({', '.join(COLUMNS)})")
    return table


def table_errors(table: np.ndarray, approximant: str) -> dict:
    """The checks of a parameter table, row by row as the reference's
    ``_validate_rows`` makes them (``_api.py:292-305``), vectorised: the
    common checks of ``check_binary`` (``_binary.py:108-126``) and the
    in-plane spins of a non-precessing approximant. ``{row: error}`` for the
    rows that fail, with the first failing check's error."""
    t = np.asarray(table, dtype=float)
    errors = {}
    m1, m2 = t[:, 0], t[:, 1]
    s1, s2 = t[:, 2:5], t[:, 5:8]
    checks = [
        (~(np.isfinite(m1) & np.isfinite(m2)) | (m1 <= 0) | (m2 <= 0), "masses must be positive"),
        (~np.all(np.isfinite(s1), axis=1) | (np.linalg.norm(s1, axis=1) > 1.0), "spin_1 must have magnitude <= 1"),
        (~np.all(np.isfinite(s2), axis=1) | (np.linalg.norm(s2, axis=1) > 1.0), "spin_2 must have magnitude <= 1"),
        (~np.isfinite(t[:, 8]) | (t[:, 8] <= 0), "luminosity_distance must be positive"),
        (~np.isfinite(t[:, 11]) | (t[:, 11] < 0), "f_ref must be positive, or zero for the model's default"),
        (~np.isfinite(t[:, 9]), "inclination must be finite"),
        (~np.isfinite(t[:, 10]), "phi_ref must be finite"),
        (np.any(s1[:, :2] != 0.0, axis=1) | np.any(s2[:, :2] != 0.0, axis=1),
         f"non-zero in-plane spins were given, but {approximant} is a non-precessing approximant"),
    ]
    for failed, message in checks:
        for i in np.flatnonzero(failed):
            errors.setdefault(int(i), InvalidParameterError(message))
    return errors


def check_binary(binary: Binary) -> None:
    """The common checks of LALSimulation on one binary of concrete values;
    raises ``InvalidParameterError`` (reference ``_binary.py:108-126``)."""
    row = np.concatenate([np.atleast_1d(np.asarray(v, dtype=float)).ravel()
                          for v in (binary.mass_1, binary.mass_2, binary.spin_1, binary.spin_2,
                                    binary.luminosity_distance, binary.inclination, binary.phi_ref, binary.f_ref)])
    error = table_errors(row[None, :12], "")
    if error and "in-plane" not in str(error[0]):
        raise error[0]


def aligned_table(table: np.ndarray) -> np.ndarray:
    """The ``(n, 8)`` parameters of the kernels from an ``(n, 12)`` table:
    the masses, the spins' z components, the distance, the inclination,
    ``phi_ref`` and ``f_ref`` (the reference's ``aligned_parameters``,
    ``models/xas/model.py:25-32``)."""
    t = np.asarray(table, dtype=np.float64)
    return np.ascontiguousarray(t[:, [0, 1, 4, 7, 8, 9, 10, 11]])
