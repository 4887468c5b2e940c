"""Write the coefficient tables of the phenomenological fits of IMRPhenomXAS
and IMRPhenomD, the numbers that define the two models (LALSimulation
6.2.0's fits, as the reference writes them), in two forms:

* ``waveformx_b200/csrc/fit_tables.h``: the C++ tables, and
  ``waveformx_b200/csrc/fit_code.h``: the same as straight-line nested
  Horner rules, which the per-binary set-up kernels evaluate;
* ``oracle/fit_tables.py``: the same tables for the CPU oracle.

Each fit becomes a sum of parts ``num(x) / den(x)`` (``den`` absent for a
polynomial), each a list of monomials ``c * prod_i x_i^e_i`` over the fit's
variables. The expansion is symbolic (sympy, in 53-bit floats) of the
reference's expressions, read from a checkout of the reference:

* ``models/xpnr/_generated/{inspiral,intermediate,ringdown}.py``: the
  collocation-point fits of the (2,2) amplitude and phase, in ``(eta, s,
  dchi, delta)``;
* ``models/xpnr/_generated/utilities.py``: ``f_meco``, ``final_mass_2017``,
  ``final_spin_2017``, ``linb`` and ``psi4_to_strain`` (their inner spin
  combination and ``sqrt(1 - 4 eta)`` as variables);
* ``models/xpnr/_generated/qnm.py``: the QNM fits, re-expanded in powers of
  ``u = 1 - a`` as ``models/xas/core.py:183-207`` does;
* ``models/xpnr/amp22.py:65-69`` and ``models/xpnr/phase22.py:295-312``:
  the TaylorF2 amplitude and phase coefficients, in ``(eta, chi1, chi2,
  delta)``;
* ``models/taylorf2/pn.py:29-91``: the TaylorF2 phasing of IMRPhenomD, in
  ``(eta, x1, x2, chi1, chi2)``;
* ``models/phenomd/core.py:129-151`` (``_amplitude_pn``) and
  ``models/phenomd/fits.py``: the amplitude PN terms, the phenomenological
  coefficients, the final spin, the radiated energy and the Chebyshev QNM
  fits.

Run from the repository root: ``python tests/golden/make_fit_tables.py``.
"""

from __future__ import annotations

import inspect
import os
import re
import sys
from pathlib import Path

import numpy as np
import sympy

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]

ETA, S, DCHI, DELTA, CHI1, CHI2, X1, X2, XI = sympy.symbols("eta s dchi delta chi1 chi2 x1 x2 xi")


def fma(a, b, c):
    return a * b + c


def _monomials(expr, variables):
    """The monomials of a polynomial: ``[(coefficient, exponents)]``."""
    poly = sympy.Poly(sympy.expand(expr), *variables)
    out = []
    for exps, coefficient in sorted(poly.terms(), key=lambda t: t[0]):
        c = float(coefficient)
        if c != 0.0:
            out.append((c, tuple(int(e) for e in exps)))
    return out


def _parts(expr, variables):
    """``expr`` (a sum of ratios of polynomials, as the fits are written) as
    parts ``(numerator monomials, denominator monomials or None)``; the
    polynomial terms are gathered into one part, placed last."""
    parts, poly = [], sympy.Integer(0)
    for term in sympy.Add.make_args(expr):
        num, den = sympy.fraction(term)
        if den == 1:
            poly = poly + term
        else:
            parts.append((_monomials(num, variables), _monomials(den, variables)))
    if poly != 0:
        parts.append((_monomials(poly, variables), None))
    return parts


def _checked(name, parts, variables, function, samples):
    """Compare the tables with the reference's function at sample points."""
    for point in samples:
        values = dict(zip(variables, point))
        x = np.array(point, dtype=float)
        total = 0.0
        for num, den in parts:
            n = sum(c * np.prod(x ** np.array(e)) for c, e in num)
            d = 1.0 if den is None else sum(c * np.prod(x ** np.array(e)) for c, e in den)
            total += n / d
        expected = float(function(values))
        assert abs(total - expected) <= 1e-12 * max(1.0, abs(expected)), (name, point, total, expected)
    return parts


def build(reference: Path):
    sys.path.insert(0, str(HERE))
    os.environ["WAVEFORMX_REFERENCE"] = str(reference)
    import reference_loader

    reference_loader.load()
    import importlib

    gen = {m: importlib.import_module(f"waveformx.models.xpnr._generated.{m}")
           for m in ("inspiral", "intermediate", "ringdown", "utilities", "qnm")}
    mathmod = importlib.import_module("waveformx.models.xpnr._math")
    amp22 = importlib.import_module("waveformx.models.xpnr.amp22")
    phase22 = importlib.import_module("waveformx.models.xpnr.phase22")
    pn = importlib.import_module("waveformx.models.taylorf2.pn")
    pd_core = importlib.import_module("waveformx.models.phenomd.core")
    pd_fits = importlib.import_module("waveformx.models.phenomd.fits")
    qnm_fit = importlib.import_module("waveformx.models.phenomd._qnm_fit")

    rng = np.random.default_rng(3)
    fits = {}  # name -> (variables names, parts)
    xas4 = (ETA, S, DCHI, DELTA)
    samples4 = [(rng.uniform(0.01, 0.25), rng.uniform(-0.9, 0.9), rng.uniform(-1.5, 1.5), rng.uniform(0, 1))
                for _ in range(4)]

    def numeric4(function):
        return lambda v: function(*(v[k] for k in xas4))

    table4 = [
        ("XAS_AMP_INS_V2", gen["inspiral"].amp_22_v2), ("XAS_AMP_INS_V3", gen["inspiral"].amp_22_v3),
        ("XAS_AMP_INS_V4", gen["inspiral"].amp_22_v4), ("XAS_PHASE_INS_V3", gen["inspiral"].phase_22_v3),
        ("XAS_PHASE_INS_D13", gen["inspiral"].phase_22_d13), ("XAS_PHASE_INS_D23", gen["inspiral"].phase_22_d23),
        ("XAS_PHASE_INS_D43", gen["inspiral"].phase_22_d43), ("XAS_AMP_INT_VA", gen["intermediate"].amp_22_va),
        ("XAS_PHASE_INT_V2", gen["intermediate"].phase_22_v2),
        ("XAS_PHASE_INT_V2M_RDV4", gen["intermediate"].phase_22_v2m_rdv4),
        ("XAS_PHASE_INT_V3M_RDV4", gen["intermediate"].phase_22_v3m_rdv4),
        ("XAS_PHASE_INT_D43", gen["intermediate"].phase_22_d43),
        ("XAS_AMP_RD_GAMMA2", gen["ringdown"].amp_22_gamma2), ("XAS_AMP_RD_GAMMA3", gen["ringdown"].amp_22_gamma3),
        ("XAS_AMP_RD_V1", gen["ringdown"].amp_22_v1), ("XAS_PHASE_RD_V4", gen["ringdown"].phase_22_v4),
        ("XAS_PHASE_RD_D12", gen["ringdown"].phase_22_d12), ("XAS_PHASE_RD_D24", gen["ringdown"].phase_22_d24),
        ("XAS_PHASE_RD_D34", gen["ringdown"].phase_22_d34), ("XAS_PHASE_RD_D54", gen["ringdown"].phase_22_d54),
        ("XAS_LINB", gen["utilities"].linb),
    ]
    for name, function in table4:
        parts = _parts(function(*xas4), xas4)
        fits[name] = ("eta s dchi delta", _checked(name, parts, xas4, numeric4(function), samples4))

    # the utilities whose spin combination and sqrt(1 - 4 eta) are computed
    # inside: patched to the variables s and delta
    util = gen["utilities"]
    saved = {k: getattr(util, k) for k in ("chi_pn_hat", "s_tot_r", "sqrt_nonneg", "jnp")}

    class _Power:
        @staticmethod
        def power(x, p):
            return x ** int(p)

    try:
        util.sqrt_nonneg = lambda x: DELTA
        util.jnp = _Power
        util.chi_pn_hat = lambda eta, c1, c2: S
        fits["XAS_F_MECO"] = ("eta s dchi delta", _parts(util.f_meco(ETA, DCHI, 0), xas4))
        util.chi_pn_hat = saved["chi_pn_hat"]
        util.s_tot_r = lambda eta, c1, c2: S
        fits["XAS_FINAL_MASS"] = ("eta s dchi delta", _parts(util.final_mass_2017(ETA, DCHI, 0), xas4))
        fits["XAS_FINAL_SPIN"] = ("eta s dchi delta", _parts(util.final_spin_2017(ETA, DCHI, 0), xas4))
        fits["XAS_PSI4_TO_STRAIN"] = ("eta s dchi delta", _parts(util.psi4_to_strain(ETA, S, DCHI), xas4))
    finally:
        for k, v in saved.items():
            setattr(util, k, v)

    # the TaylorF2 coefficients of the (2,2) amplitude and phase, in (eta,
    # chi1, chi2, delta)
    pnvars = (ETA, CHI1, CHI2, DELTA)
    pi = mathmod.POWERS_OF_LALPI
    namespace = dict(fma=fma, pi=pi, PI=mathmod.PI, EGAMMA=mathmod.EGAMMA, LN_2=mathmod.LN_2, eta=ETA, delta=DELTA,
                     chi1l=CHI1, chi2l=CHI2, eta2=ETA ** 2, eta3=ETA ** 3, chi1l2=CHI1 ** 2, chi1l3=CHI1 ** 3,
                     chi2l2=CHI2 ** 2, chi2l3=CHI2 ** 3, chi1l2l=CHI1 * CHI2)
    for module, first, last in ((amp22, "pn_two_thirds", "pn_six_thirds"), (phase22, "phi2_ns", "phi8l_s")):
        lines = inspect.getsource(module).splitlines()
        start = next(i for i, line in enumerate(lines) if line.strip().startswith(first + " ="))
        stop = next(i for i, line in enumerate(lines) if line.strip().startswith(last + " ="))
        for line in lines[start:stop + 1]:
            exec(line.strip(), namespace)  # noqa: S102 (the reference's own expressions, symbolically)
    phase_terms = dict(phi2=namespace["phi2_ns"], phi3=namespace["phi3_ns"] + namespace["phi3_s"],
                       phi4=namespace["phi4_ns"] + namespace["phi4_s"],
                       phi5l=namespace["phi5l_ns"] + namespace["phi5l_s"],
                       phi6=namespace["phi6_ns"] + namespace["phi6_s"], phi6l=namespace["phi6l_ns"],
                       phi7=namespace["phi7_ns"] + namespace["phi7_s"], phi8=namespace["phi8_s"],
                       phi8l=namespace["phi8l_s"])
    for key in ("pn_two_thirds", "pn_three_thirds", "pn_four_thirds", "pn_five_thirds", "pn_six_thirds"):
        fits["XAS_AMP_" + key.upper()] = ("eta chi1 chi2 delta", [(_monomials(namespace[key], pnvars), None)])
    for key, value in phase_terms.items():
        fits["XAS_PHASE_" + key.upper()] = ("eta chi1 chi2 delta", [(_monomials(sympy.sympify(value), pnvars), None)])

    # IMRPhenomD: TaylorF2 phasing terms (before the factor 3 / (128 eta)),
    # in (eta, x1, x2, chi1, chi2)
    pdvars = (ETA, X1, X2, CHI1, CHI2)
    fits["PHD_PN_PHASE_3"] = ("eta x1 x2 chi1 chi2", [(_monomials(pn._phase_3(X1, X2, CHI1, CHI2), pdvars), None)])
    for k, function in ((4, pn._phase_4), (5, pn._phase_5), (6, pn._phase_6), (7, pn._phase_7)):
        fits[f"PHD_PN_PHASE_{k}"] = ("eta x1 x2 chi1 chi2",
                                     [(_monomials(function(ETA, X1, X2, CHI1, CHI2), pdvars), None)])
    fits["PHD_PN_SPIN_SPIN_3"] = ("eta x1 x2 chi1 chi2",
                                  [(_monomials(pn.spin_spin_3pn(ETA, X1, X2, CHI1, CHI2), pdvars), None)])
    ampvars = (ETA, DELTA, CHI1, CHI2)
    amp_pn = pd_core._amplitude_pn(ETA, DELTA, CHI1, CHI2)
    for k in (2, 3, 4, 5, 6):
        fits[f"PHD_AMP_PN_{k}"] = ("eta delta chi1 chi2", [(_monomials(sympy.sympify(amp_pn[k]), ampvars), None)])
    # the phenomenological coefficients: sum_i xi^i sum_j c_ij eta^j
    for name, rows in pd_fits.COEFFICIENTS.items():
        terms = [(float(c), (j, i)) for i, row in enumerate(rows) for j, c in enumerate(row) if c != 0.0]
        fits["PHD_" + name.upper()] = ("eta xi", [(terms, None)])
    terms = [(float(c), (j, i)) for i, row in enumerate(pd_fits._FINAL_SPIN) for j, c in enumerate(row) if c != 0.0]
    fits["PHD_FINAL_SPIN"] = ("eta s", [(terms, None)])
    # the radiated energy, with its spin combination as the variable s
    energy = pd_fits.radiated_energy(ETA, 0, S, S)
    num, den = sympy.fraction(sympy.together(energy))
    num_m, den_m = _monomials(num, (ETA, S)), _monomials(den, (ETA, S))
    # (normalise the constant of the denominator to one, as the fit is written)
    d0 = dict((e, c) for c, e in den_m)[(0, 0)]
    fits["PHD_RADIATED_ENERGY"] = ("eta s", [([(c / d0, e) for c, e in num_m], [(c / d0, e) for c, e in den_m])])

    # the QNM fits of XAS re-expanded about a = 1 (models/xas/core.py:183-207)
    A = sympy.symbols("a")
    qnm = {}
    for name, function in (("FRING", gen["qnm"].fring22), ("FDAMP", gen["qnm"].fdamp22)):
        num, den = sympy.fraction(function(A))
        out = []
        for poly in (num, den):
            coefficients = [float(c) for c in reversed(sympy.Poly(sympy.expand(poly), A).all_coeffs())]
            about = np.zeros(len(coefficients))
            for k, c in enumerate(coefficients):
                about[:k + 1] += c * np.polynomial.polynomial.polypow([1.0, -1.0], k)
            out.append([float(x) for x in about])
        qnm[name] = out
    chebyshev = dict(FRING=[float(x) for x in qnm_fit.FRING], FDAMP=[float(x) for x in qnm_fit.FDAMP])
    # constants the set-up uses, computed as the reference computes them (so
    # that cbrt, sqrt and pow of the host library fix their last bits once)
    xas_core = importlib.import_module("waveformx.models.xas.core")
    constants = {
        "PI": mathmod.PI, "MTSUN_SI": mathmod.MTSUN_SI, "MRSUN_SI": mathmod.MRSUN_SI, "MPC_SI": mathmod.MPC_SI,
        "EGAMMA": mathmod.EGAMMA, "LN_2": mathmod.LN_2,
        "LALPI_ONE_SIXTH": pi.one_sixth, "LALPI_M_ONE_SIXTH": pi.m_one_sixth, "LALPI_ONE_THIRD": pi.one_third,
        "LALPI_TWO_THIRDS": pi.two_thirds, "LALPI_FOUR_THIRDS": pi.four_thirds, "LALPI_FIVE_THIRDS": pi.five_thirds,
        "LALPI_M_FIVE_THIRDS": pi.m_five_thirds, "LALPI_SEVEN_THIRDS": pi.seven_thirds,
        "LALPI_EIGHT_THIRDS": pi.eight_thirds, "LALPI_TWO": pi.two, "LALPI_LOG": pi.log,
        "XAS_K0": xas_core.K0, "XAS_YLM": xas_core.YLM, "PHD_K_AMP": pd_core.K_AMP,
        "SQRT_TWO_THIRDS": float(np.sqrt(2.0 / 3.0)),
        "PI_POW_4_3": mathmod.PI ** (4.0 / 3.0), "PI_POW_5_3": mathmod.PI ** (5.0 / 3.0),
        "PI_POW_7_3": mathmod.PI ** (7.0 / 3.0), "PI_POW_8_3": mathmod.PI ** (8.0 / 3.0),
        "PI_POW_2": mathmod.PI ** 2, "PI_POW_3": mathmod.PI ** 3,
        "XAS_DPHASE0": 5.0 / (128.0 * mathmod.PI ** (5.0 / 3.0)),
    }
    return fits, qnm, chebyshev, {k: float(v) for k, v in constants.items()}


def _c_double(x):
    return repr(float(x))


def write_header(path, fits, qnm, chebyshev, constants):
    names = list(fits)
    terms, parts, firsts = [], [], []
    for name in names:
        _, fit_parts = fits[name]
        firsts.append((len(parts), len(fit_parts)))
        for num, den in fit_parts:
            begin = len(terms)
            terms.extend(num)
            den_begin = len(terms)
            if den is not None:
                terms.extend(den)
            parts.append((begin, len(num), den_begin, 0 if den is None else len(den)))
    lines = [
        "// GENERATED by tests/golden/make_fit_tables.py: the coefficients of the",
        "// phenomenological fits of IMRPhenomXAS and IMRPhenomD (LALSimulation 6.2.0's",
        "// fits, which define the two models) as monomial tables; do not edit.",
        "#pragma once",
        "",
        "namespace wfx {",
        "namespace fit {",
        "",
        "// One monomial c * prod_i x_i^e[i] of a fit's variables.",
        "struct Term {",
        "  double c;",
        "  signed char e[6];",
        "};",
        "",
        "// A part num(x) / den(x) of a fit (den_count == 0: den = 1).",
        "struct Part {",
        "  short num_begin, num_count, den_begin, den_count;",
        "};",
        "",
        "// A fit: the sum of its parts, in order.",
        "struct Fit {",
        "  short part_begin, part_count;",
        "};",
        "",
        "enum Id : int {",
    ]
    for i, name in enumerate(names):
        lines.append(f"  {name} = {i},  // variables: {fits[name][0]}")
    lines += [f"  COUNT = {len(names)}", "};", ""]
    lines.append("#define WFX_FIT_TERMS \\")
    lines.append("  { \\")
    for c, e in terms:
        e = tuple(e) + (0,) * (6 - len(e))
        lines.append(f"    {{{_c_double(c)}, {{{', '.join(str(x) for x in e)}}}}}, \\")
    lines.append("  }")
    lines.append("")
    lines.append("#define WFX_FIT_PARTS \\")
    lines.append("  { \\")
    for p in parts:
        lines.append(f"    {{{p[0]}, {p[1]}, {p[2]}, {p[3]}}}, \\")
    lines.append("  }")
    lines.append("")
    lines.append("#define WFX_FIT_FITS \\")
    lines.append("  { \\")
    for b, n in firsts:
        lines.append(f"    {{{b}, {n}}}, \\")
    lines.append("  }")
    lines.append("")
    lines.append(f"constexpr int kTermCount = {len(terms)};")
    lines.append(f"constexpr int kPartCount = {len(parts)};")
    lines.append("")
    lines.append("// The (2,2) QNM fits of IMRPhenomXAS, numerator and denominator in powers")
    lines.append("// of u = 1 - a_final (lowest first).")
    for name, (num, den) in qnm.items():
        lines.append(f"#define WFX_XAS_{name}_NUM {{{', '.join(_c_double(x) for x in num)}}}")
        lines.append(f"#define WFX_XAS_{name}_DEN {{{', '.join(_c_double(x) for x in den)}}}")
        lines.append(f"constexpr int kXas{name.title()}NumCount = {len(num)};")
        lines.append(f"constexpr int kXas{name.title()}DenCount = {len(den)};")
    lines.append("")
    lines.append("// The (2,2) QNM fits of IMRPhenomD: Chebyshev series (lowest degree first) in")
    lines.append("// t = 2 ((1 - a_final) / 2)^(1/3) - 1.")
    for name, values in chebyshev.items():
        lines.append(f"#define WFX_PHD_{name} {{{', '.join(_c_double(x) for x in values)}}}")
    lines.append(f"constexpr int kPhdChebyshevCount = {len(chebyshev['FRING'])};")
    lines.append("")
    lines.append("// Constants of the set-up (doubles as the reference computes them).")
    for name, value in constants.items():
        lines.append(f"constexpr double {name} = {_c_double(value)};")
    lines += ["", "}  // namespace fit", "}  // namespace wfx", ""]
    path.write_text("\n".join(lines))


def _horner_code(terms, nvars, var=0):
    """C++ of sum_t c_t prod_i x_i^e_ti by nested Horner rules: in x_var,
    whose coefficients are polynomials in the later variables."""
    if var == nvars:
        return _c_double(sum(c for c, _ in terms))
    by_power = {}
    for c, e in terms:
        by_power.setdefault(e[var], []).append((c, e))
    top = max(by_power)
    code = None
    for k in range(top, -1, -1):
        inner = _horner_code(by_power[k], nvars, var + 1) if k in by_power else None
        if code is None:
            code = f"R({inner})" if inner and not inner.startswith("(") and var + 1 == nvars else inner
        else:
            code = f"({code}) * x{var}" + (f" + {inner}" if inner is not None else "")
    return code


def write_code(path, fits):
    """Straight-line C++ of every fit (nested Horner rules), for the set-up
    kernels: ``fit_<NAME>(x0, ...)`` and the dispatcher ``fit_call<R>(id, x)``."""
    lines = [
        "// GENERATED by tests/golden/make_fit_tables.py from the fit tables of",
        "// fit_tables.h (LALSimulation 6.2.0's IMRPhenomXAS and IMRPhenomD fits) as",
        "// straight-line nested Horner rules; do not edit.",
        "#pragma once",
        "",
        '#include "fit_tables.h"',
        '#include "scalar.cuh"',
        "",
        "namespace wfx {",
        "namespace fit {",
        "",
    ]
    names = list(fits)
    for name in names:
        variables, parts = fits[name]
        nv = len(variables.split())
        args = ", ".join(f"const R& x{i}" for i in range(nv))
        lines.append(f"// {name}({variables})")
        lines.append(f"template <class R>")
        lines.append(f"WFX_HD R fit_{name.lower()}({args}) {{")
        exprs = []
        for j, (num, den) in enumerate(parts):
            n = _horner_code(num, nv)
            lines.append(f"  const R n{j} = {n};")
            if den is not None:
                d = _horner_code(den, nv)
                lines.append(f"  const R d{j} = {d};")
                exprs.append(f"n{j} / d{j}")
            else:
                exprs.append(f"n{j}")
        total = exprs[0]
        for e in exprs[1:]:
            total = f"({total}) + {e}"
        lines.append(f"  return {total};")
        lines.append("}")
        lines.append("")
    lines.append("// The fit `id` at x[0 .. nvars): a switch that folds where id is a constant.")
    lines.append("template <class R>")
    lines.append("WFX_HD R fit_call(int id, const R* x) {")
    lines.append("  switch (id) {")
    for name in names:
        nv = len(fits[name][0].split())
        args = ", ".join(f"x[{i}]" for i in range(nv))
        lines.append(f"    case {name}:")
        lines.append(f"      return fit_{name.lower()}({args});")
    lines.append("    default:")
    lines.append("      return R(NAN);")
    lines.append("  }")
    lines.append("}")
    lines += ["", "}  // namespace fit", "}  // namespace wfx", ""]
    path.write_text("\n".join(lines))


def write_python(path, fits, qnm, chebyshev, constants):
    lines = [
        '"""GENERATED by tests/golden/make_fit_tables.py: the coefficients of the',
        "phenomenological fits of IMRPhenomXAS and IMRPhenomD (LALSimulation 6.2.0's",
        "fits, which define the two models) as monomial tables, for the oracle;",
        'do not edit.',
        "",
        "``FITS[name] = (variables, parts)``; a part is ``(numerator, denominator)``,",
        "each a list of ``(coefficient, exponents)`` (``denominator`` None: one).",
        '"""',
        "",
        "FITS = {",
    ]
    for name, (variables, parts) in fits.items():
        lines.append(f"    {name!r}: ({variables!r}, [")
        for num, den in parts:
            lines.append(f"        ({[(c, e) for c, e in num]!r},")
            lines.append(f"         {None if den is None else [(c, e) for c, e in den]!r}),")
        lines.append("    ]),")
    lines.append("}")
    lines.append("")
    lines.append("# the (2,2) QNM fits of IMRPhenomXAS in powers of u = 1 - a (numerator, denominator)")
    for name, (num, den) in qnm.items():
        lines.append(f"XAS_{name} = ({num!r}, {den!r})")
    lines.append("")
    lines.append("# the (2,2) QNM fits of IMRPhenomD: Chebyshev coefficients in t = 2 ((1 - a) / 2)^(1/3) - 1")
    for name, values in chebyshev.items():
        lines.append(f"PHD_{name} = {values!r}")
    lines.append("")
    lines.append("# constants of the set-up, as the reference computes them")
    lines.append(f"CONSTANTS = {constants!r}")
    lines.append("")
    path.write_text("\n".join(lines))


def main():
    if not os.environ.get("WAVEFORMX_REFERENCE"):
        raise SystemExit("set WAVEFORMX_REFERENCE to the reference checkout's root")
    reference = Path(os.environ["WAVEFORMX_REFERENCE"])
    fits, qnm, chebyshev, constants = build(reference)
    write_header(ROOT / "waveformx_b200" / "csrc" / "fit_tables.h", fits, qnm, chebyshev, constants)
    write_code(ROOT / "waveformx_b200" / "csrc" / "fit_code.h", fits)
    write_python(ROOT / "oracle" / "fit_tables.py", fits, qnm, chebyshev, constants)
    print(f"{len(fits)} fits, {sum(len(n) + len(d or []) for _, p in fits.values() for n, d in p)} monomials")


if __name__ == "__main__":
    main()
