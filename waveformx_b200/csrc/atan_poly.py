"""The coefficients of the FP32 kernels' arctangent (``m_atan`` in
``point.cuh``): atan(x) ~ x P(x^2) on [0, 1], P of degree 6, minimax in the
absolute error by the Remez exchange algorithm; |x| > 1 is reduced by
atan(x) = pi/2 - atan(1/x). Prints the float32 coefficients and the maximum
error of the float32-rounded polynomial (about 2.5e-7).

    python waveformx_b200/csrc/atan_poly.py
"""

import numpy as np


def remez(degree, iterations=30, grid=200001):
    n = degree + 1
    k = np.arange(n + 1)
    x = 0.5 - 0.5 * np.cos(np.pi * k / n)
    x[0] = 1e-6
    xs = np.linspace(0.0, 1.0, grid)
    for _ in range(iterations):
        a = np.column_stack([x * (x * x) ** j for j in range(n)] + [(-1.0) ** k])
        coef = np.linalg.solve(a, np.arctan(x))[:n]
        err = xs * np.polyval(coef[::-1], xs * xs) - np.arctan(xs)
        d = np.diff(err)
        cand = np.concatenate([[0], np.where(np.sign(d[:-1]) != np.sign(d[1:]))[0] + 1, [grid - 1]])
        while len(cand) > n + 1:
            vals = np.abs(err[cand])
            for i in range(len(cand) - 1):
                if np.sign(err[cand[i]]) == np.sign(err[cand[i + 1]]):
                    cand = np.delete(cand, i if vals[i] < vals[i + 1] else i + 1)
                    break
            else:
                cand = np.delete(cand, 0 if vals[0] < vals[-1] else len(cand) - 1)
        x = xs[cand]
        x[0] = max(x[0], 1e-6)
    return coef


if __name__ == "__main__":
    c32 = remez(6).astype(np.float32)
    xs = np.linspace(0.0, 1.0, 1000001)
    err = xs * np.polyval(c32.astype(np.float64)[::-1], xs * xs) - np.arctan(xs)
    print("coefficients of s^0 .. s^6:", ", ".join(f"{float(c):.9e}f" for c in c32))
    print("max |error| on [0, 1]:", np.max(np.abs(err)))
