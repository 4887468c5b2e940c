"""Write ``waveformx_b200/csrc/hm_fit_code.h``: the phenomenological fits of
the higher modes of IMRPhenomXHM (LALSimulation 6.2.0's fits, release
122022, which define the model) as straight-line nested Horner rules, for
the per-binary set-up kernels; and the QNM and mixing-coefficient fits of
the higher modes re-expanded in powers of ``u = 1 - a_final``, as
``models/xhm/reference.py:98-99`` uses them (``models/xas/core.py:191-207``).

Each fit of the reference's generated modules
(``models/xpnr/_generated/hm_amp_fits_{inspiral,intermediate,ringdown}.py``,
``hm_intermediate.py``, ``hm_inspiral.py``, ``hm_ringdown.py``) is called
with symbols for the binary's variables (``eta`` written as ``sq^2``, ``sq
= sqrt(eta)``; ``delta = sqrt(1 - 4 eta)`` and ``r3 = sqrt(1 - 3 eta)``
symbols of their own), expanded (sympy, 53-bit floats) into a sum of
ratios of polynomials and checked against the reference's own function at
sample points. A fit the reference wraps in ``abs`` is written without it
(the set-up applies it). The fits of ``hm_ringdown.py`` are prefixed
``rd_`` (its ``phase_32_p1`` ... are not those of ``hm_intermediate.py``). Variables of the generated functions, in this
order: ``sq delta r3 s dh dc st c1 c2`` = ``sqrt(eta)``, ``delta``,
``sqrt(1 - 3 eta)``, ``chi_pn_hat``, ``dchi_half``, ``dchi``, ``s_tot_r``,
``chi1l``, ``chi2l``.

Run from the repository root: ``python tests/golden/make_hm_fit_code.py``.
"""

from __future__ import annotations

import importlib
import inspect
import os
import re
import sys
from pathlib import Path

import numpy as np
import sympy

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(HERE))
from make_fit_tables import _c_double, _horner_code, _parts  # noqa: E402

SQ, DELTA, R3, S, DH, DC, ST, C1, C2 = sympy.symbols("sq delta r3 s dh dc st c1 c2", real=True)
SQ = sympy.Symbol("sq", positive=True)
VARIABLES = (SQ, DELTA, R3, S, DH, DC, ST, C1, C2)
NAMES = ("sq", "delta", "r3", "s", "dh", "dc", "st", "c1", "c2")
ETA = SQ ** 2
ABS = sympy.Function("ABS")


class _Wf:
    """The binary's variables as symbols (or numbers, for the checks)."""

    def __init__(self, values):
        self.__dict__.update(values)


def _symbolic_wf():
    return _Wf(dict(eta=ETA, delta=DELTA, chi_pn_hat=S, dchi_half=DH, dchi=DC, s_tot_r=ST, chi1l=C1, chi2l=C2))


class _Jnp:
    """``jax.numpy`` for the symbolic call: the roots the fits take (of eta,
    1 - 3 eta and their products with eta), integer and half-integer powers,
    and abs."""

    @staticmethod
    def sqrt(x):
        for form, root in ((ETA, SQ), (1 - 3 * ETA, R3), (ETA - 3 * ETA ** 2, SQ * R3)):
            if sympy.simplify(sympy.expand(x - form)) == 0:
                return root
        raise ValueError(f"sqrt of {x}")

    @staticmethod
    def power(x, p):
        return x ** sympy.Rational(p).limit_denominator(8)

    @staticmethod
    def abs(x):
        return ABS(x)


def _sqrt_nonneg(x):
    for form, root in ((1 - 4 * ETA, DELTA), (ETA - 4 * ETA ** 2, SQ * DELTA)):
        if sympy.simplify(sympy.expand(x - form)) == 0:
            return root
    raise ValueError(f"sqrt_nonneg of {x}")


def _symbolic(module, function):
    saved = {k: getattr(module, k) for k in ("jnp", "sqrt_nonneg") if hasattr(module, k)}
    try:
        module.jnp = _Jnp
        module.sqrt_nonneg = _sqrt_nonneg
        expr = function(_symbolic_wf())
    finally:
        for k, v in saved.items():
            setattr(module, k, v)
    wrapped = isinstance(expr, ABS)
    if wrapped:
        expr = expr.args[0]
    assert not expr.has(ABS), function.__name__
    return sympy.sympify(expr), wrapped


def _evaluate(parts, variables, x):
    total = 0.0
    for num, den in parts:
        n = sum(c * np.prod([x[v] ** e for v, e in zip(variables, ex)]) for c, ex in num)
        d = 1.0 if den is None else sum(c * np.prod([x[v] ** e for v, e in zip(variables, ex)]) for c, ex in den)
        total += n / d
    return total


def build():
    import reference_loader

    reference_loader.load()
    gen = {m: importlib.import_module(f"waveformx.models.xpnr._generated.{m}")
           for m in ("hm_amp_fits_inspiral", "hm_amp_fits_intermediate", "hm_amp_fits_ringdown", "hm_intermediate",
                     "hm_inspiral", "hm_ringdown", "hm_qnm")}
    rng = np.random.default_rng(5)
    samples = []
    for _ in range(4):
        eta = rng.uniform(0.01, 0.249)
        samples.append(dict(eta=eta, delta=np.sqrt(1 - 4 * eta), chi_pn_hat=rng.uniform(-0.9, 0.9),
                            dchi_half=rng.uniform(-0.9, 0.9), dchi=rng.uniform(-1.5, 1.5),
                            s_tot_r=rng.uniform(-0.9, 0.9), chi1l=rng.uniform(-0.9, 0.9), chi2l=rng.uniform(-0.9, 0.9)))
    fits = {}
    patterns = {
        "hm_amp_fits_inspiral": r"amp_\d\d_iv\d$", "hm_amp_fits_intermediate": r"amp_\d\d_int\d$",
        "hm_amp_fits_ringdown": r"amp_\d\d_\w+$", "hm_intermediate": r"phase_\d\d_p\d$",
        "hm_inspiral": r"phase_\d\d_lambda$",
        "hm_ringdown": r"phase_(32_p\d|22_alpha2|22_alpha_l|32_spheroidal_time_shift|32_spheroidal_phase_shift)$",
    }
    for module_name, pattern in patterns.items():
        module = gen[module_name]
        for name, function in inspect.getmembers(module, inspect.isfunction):
            if function.__module__ != module.__name__ or not re.match(pattern, name):
                continue
            expr, wrapped = _symbolic(module, function)
            used = [v for v in VARIABLES if expr.has(v)]
            parts = _parts(expr, used)
            for point in samples:
                x = {SQ: np.sqrt(point["eta"]), DELTA: point["delta"], R3: np.sqrt(1 - 3 * point["eta"]),
                     S: point["chi_pn_hat"], DH: point["dchi_half"], DC: point["dchi"], ST: point["s_tot_r"],
                     C1: point["chi1l"], C2: point["chi2l"]}
                got = _evaluate(parts, used, x)
                if wrapped:
                    got = abs(got)
                expected = float(function(_Wf(point)))
                assert abs(got - expected) <= 1e-11 * max(1.0, abs(expected)), (name, got, expected)
            # (hm_ringdown's phase_32_p* differ from hm_intermediate's: prefixed)
            key = ("rd_" if module_name == "hm_ringdown" else "") + name
            assert key not in fits, key
            fits[key] = ([NAMES[VARIABLES.index(v)] for v in used], parts, wrapped)
    # the QNM and mixing fits of the higher modes, about a = 1
    a = sympy.symbols("a")
    qnm = {}
    module = gen["hm_qnm"]
    for name, function in inspect.getmembers(module, inspect.isfunction):
        if function.__module__ != module.__name__ or not name.startswith(("fring", "fdamp", "re_l", "im_l")):
            continue
        num, den = sympy.fraction(sympy.together(function(a)))
        out = []
        for poly in (num, den):
            coefficients = [float(c) for c in reversed(sympy.Poly(sympy.expand(poly), a).all_coeffs())]
            about = np.zeros(len(coefficients))
            for k, c in enumerate(coefficients):
                about[:k + 1] += c * np.polynomial.polynomial.polypow([1.0, -1.0], k)
            out.append([float(x) for x in about])
        # (normalise the constant of the denominator to one)
        d0 = out[1][0]
        out = [[x / d0 for x in out[0]], [x / d0 for x in out[1]]]
        for spin in (-0.9, 0.0, 0.7, 0.99):
            u = 1.0 - spin
            got = np.polynomial.polynomial.polyval(u, out[0]) / np.polynomial.polynomial.polyval(u, out[1])
            expected = float(function(spin))
            assert abs(got - expected) <= 1e-11 * max(1.0, abs(expected)), (name, spin, got, expected)
        qnm[name] = out
    return fits, qnm


def write(path, fits, qnm):
    lines = [
        "// GENERATED by tests/golden/make_hm_fit_code.py: the phenomenological fits of",
        "// the higher modes of IMRPhenomXHM (LALSimulation 6.2.0, release 122022) as",
        "// straight-line nested Horner rules, and their QNM and mixing fits in powers",
        "// of u = 1 - a_final; do not edit.",
        "#pragma once",
        "",
        '#include "scalar.cuh"',
        "",
        "namespace wfx {",
        "namespace hmfit {",
        "",
        "// The variables of the fits: sqrt(eta), delta = sqrt(1 - 4 eta),",
        "// sqrt(1 - 3 eta), chi_pn_hat, dchi_half, dchi, s_tot_r, chi1, chi2.",
        "template <class R>",
        "struct Args {",
        "  R sq, delta, r3, s, dh, dc, st, c1, c2;",
        "};",
        "",
    ]
    for name, (names, parts, wrapped) in fits.items():
        nv = len(names)
        lines.append(f"// {name}({', '.join(names)})" + ("  (the reference takes its absolute value)" if wrapped else ""))
        lines.append("template <class R>")
        lines.append(f"WFX_HD R {name}(const Args<R>& a) {{")
        exprs = []
        for j, (num, den) in enumerate(parts):
            n = _horner_code(num, nv) if nv else _c_double(sum(c for c, _ in num))
            n = re.sub(r"\bx(\d)\b", lambda m: f"a.{names[int(m.group(1))]}", n)
            lines.append(f"  const R n{j} = {n if nv else f'R({n})'};")
            if den is not None:
                d = _horner_code(den, nv) if nv else _c_double(sum(c for c, _ in den))
                d = re.sub(r"\bx(\d)\b", lambda m: f"a.{names[int(m.group(1))]}", d)
                lines.append(f"  const R d{j} = {d if nv else f'R({d})'};")
                exprs.append(f"n{j} / d{j}")
            else:
                exprs.append(f"n{j}")
        total = exprs[0]
        for e in exprs[1:]:
            total = f"({total}) + {e}"
        lines.append(f"  return {total};")
        lines.append("}")
        lines.append("")
    lines.append("// QNM and mixing fits of the final spin a, as ratios of polynomials in")
    lines.append("// u = 1 - a (Horner rules; the denominator's constant one).")

    def horner(coefficients):
        code = _c_double(coefficients[-1])
        for c in coefficients[-2::-1]:
            code = f"({code}) * u + {_c_double(c)}"
        return code

    for name, (num, den) in qnm.items():
        lines.append("template <class R>")
        lines.append(f"WFX_HD R {name}(const R& a) {{")
        lines.append("  const R u = 1.0 - a;")
        lines.append(f"  return ({horner(num)}) /")
        lines.append(f"         ({horner(den)});")
        lines.append("}")
    lines += ["", "}  // namespace hmfit", "}  // namespace wfx", ""]
    path.write_text("\n".join(lines))


def main():
    if not os.environ.get("WAVEFORMX_REFERENCE"):
        raise SystemExit("set WAVEFORMX_REFERENCE to the reference checkout's root")
    fits, qnm = build()
    out = ROOT / "waveformx_b200" / "csrc" / "hm_fit_code.h"
    write(out, fits, qnm)
    print(f"{out}: {len(fits)} fits, {len(qnm)} QNM fits")


if __name__ == "__main__":
    main()
