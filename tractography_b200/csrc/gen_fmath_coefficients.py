"""Polynomial coefficients of the step's specialised functions in tg_fmath.h.

Each polynomial is fitted to the relative error of its function by least
squares on 4000 Chebyshev nodes, the weights raised where the error is
largest and the fit repeated (Lawson's iteration towards the minimax
polynomial); the coefficients are then rounded to binary32.

  log   tgm_log_pos: log(1 + f) = f - f^2/2 + f^3 Q(f), f in [sqrt(1/2) - 1,
        sqrt(2) - 1], Q of degree 7 (relative error of the fit ~2^-27.4).
  sin   tgm_cos2pi_u24: sin(t) = t + t^3 S(t^2), |t| <= pi/4, S of degree 2
        (~2^-28).
  cos   tgm_cos2pi_u24: cos(t) = 1 + t^2 C(t^2), |t| <= pi/4, C of degree 3
        (~2^-33.9).
  expc  tgm_exps2_factors: cos(n) = 1 + n2 P(n2), n2 = n^2 in [0, 1), P of
        degree 3 (~2^-30.2).
  expk  tgm_exps2_factors: sin(n)/n = 1 + n2 K(n2), n2 in [0, 1), K of
        degree 3 (~2^-34).

Evaluated in binary32 with fused multiply-adds as tg_fmath.h does, the
results stay within the ulp bounds tests/test_math.py checks.

    python gen_fmath_coefficients.py    # prints every coefficient
"""

import numpy as np


def _nodes(a: float, b: float, n: int = 4000):
    t = np.cos(np.pi * (np.arange(n) + 0.5) / n)
    return (a + b) / 2 + (b - a) / 2 * t


def _lawson(x, target, degree: int, scale, iterations: int = 80):
    basis = np.vander(x, degree + 1, increasing=True)
    weights = np.ones(len(x))
    for _ in range(iterations):
        coef, *_ = np.linalg.lstsq(basis * (scale * weights)[:, None], target * scale * weights, rcond=None)
        err = np.abs(basis @ coef - target) * scale
        weights *= np.sqrt(err / err.max()) + 1e-3
    return coef.astype(np.float32), float(err.max())


def fit(name: str = "log"):
    """(binary32 coefficients in increasing degree, relative error of the float64 fit)."""
    if name == "log":
        f = _nodes(np.sqrt(0.5) - 1.0, np.sqrt(2.0) - 1.0)
        y = np.log1p(f)
        return _lawson(f, (y - f + f * f / 2) / f**3, 7, np.abs(f**3 / y), iterations=60)
    if name in ("sin", "cos"):
        x = _nodes(1e-12, (np.pi / 4) ** 2)
        t = np.sqrt(x)
        if name == "sin":
            return _lawson(x, (np.sin(t) - t) / t**3, 2, t**3 / np.sin(t))
        return _lawson(x, (np.cos(t) - 1) / x, 3, x / np.cos(t))
    if name in ("expc", "expk"):
        x = _nodes(1e-12, 1.0)
        n = np.sqrt(x)
        y = np.cos(n) if name == "expc" else np.sin(n) / n
        return _lawson(x, (y - 1) / x, 3, x / y)
    raise ValueError(name)


if __name__ == "__main__":
    for name in ("log", "sin", "cos", "expc", "expk"):
        q, err = fit(name)
        print(f"{name}: relative error of the float64 fit {err:.3e}")
        for k, c in enumerate(q):
            print(f"  {k}: {float(c).hex()}f")
