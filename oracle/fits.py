"""Evaluation of the monomial tables of ``fit_tables.py`` (the fits of
IMRPhenomXAS and IMRPhenomD) on arrays. Oracle only."""

from __future__ import annotations

import numpy as np

from .fit_tables import FITS


def _poly(terms, powers):
    total = 0.0
    for c, exps in terms:
        term = c
        for p, e in zip(powers, exps):
            if e:
                term = term * p[e]
        total = total + term
    return total


def evaluate(name, *variables):
    """The fit ``name`` at the arrays ``variables`` (in the order of its
    variable list)."""
    _, parts = FITS[name]
    top = max(max((max(e) for _, e in num), default=0) for num, _ in parts)
    top = max(top, max((max((max(e) for _, e in den), default=0) for _, den in parts if den), default=0))
    powers = []
    for x in variables:
        x = np.asarray(x, dtype=np.float64)
        p = [np.ones_like(x), x]
        for _ in range(top - 1):
            p.append(p[-1] * x)
        powers.append(p)
    total = 0.0
    for num, den in parts:
        value = _poly(num, powers)
        if den is not None:
            value = value / _poly(den, powers)
        total = total + value
    return total
