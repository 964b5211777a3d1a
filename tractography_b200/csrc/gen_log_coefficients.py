"""Coefficients of tgm_log_pos (tg_fmath.h): log(1 + f) = f - f^2/2 + f^3 Q(f)
for f in [sqrt(1/2) - 1, sqrt(2) - 1], Q a polynomial of degree 7.

Q is fitted to the relative error of log(1 + f) by least squares on 4000
Chebyshev nodes, the weights raised where the error is largest and the fit
repeated (Lawson's iteration towards the minimax polynomial); the
coefficients are then rounded to binary32.  The float64 fit reaches a
relative error of about 2^-27.4 in log(1 + f); evaluated in binary32 with
fused multiply-adds as tgm_log_pos does, the result stays within one ulp of
the correctly rounded logarithm over the positive normal floats checked by
tests/test_math.py.

    python gen_log_coefficients.py      # prints the eight coefficients
"""

import numpy as np


def fit(degree: int = 7, nodes: int = 4000, iterations: int = 60):
    a, b = np.sqrt(0.5) - 1.0, np.sqrt(2.0) - 1.0
    t = np.cos(np.pi * (np.arange(nodes) + 0.5) / nodes)
    f = (a + b) / 2 + (b - a) / 2 * t
    y = np.log1p(f)
    target = (y - f + f * f / 2) / f**3
    scale = np.abs(f**3 / y)              # an error in Q, relative to log(1 + f)
    weights = np.ones(nodes)
    basis = np.vander(f, degree + 1, increasing=True)
    for _ in range(iterations):
        coef, *_ = np.linalg.lstsq(basis * (scale * weights)[:, None], target * scale * weights, rcond=None)
        err = np.abs(basis @ coef - target) * scale
        weights *= np.sqrt(err / err.max()) + 1e-3
    return coef.astype(np.float32), float(err.max())


if __name__ == "__main__":
    q, err = fit()
    print(f"relative error of the float64 fit: {err:.3e}")
    for k, c in enumerate(q):
        print(f"Q{k} = {float(c).hex()}f")
