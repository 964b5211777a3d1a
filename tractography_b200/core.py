"""Host-side spherical helpers (reference ``tractography/core.py:1-95``).

These are float64 NumPy utilities used to build synthetic fields, fit
spherical-harmonic coefficients and check results; the tracking kernels do
not call them.
"""

from __future__ import annotations

import numpy as np
import scipy.special


def cart2sph(x, y, z):
    """Cartesian to (azimuth in [0, 2 pi), colatitude in [0, pi], radius).

    At the origin both angles and the radius are zero (core.py:1-30).
    """
    x, y, z = np.broadcast_arrays(x, y, z)
    radius = np.sqrt(x ** 2 + y ** 2 + z ** 2)
    nonzero = radius > 0
    cos_colatitude = np.divide(
        z, radius, out=np.zeros_like(radius, dtype=np.result_type(radius, np.float32)), where=nonzero
    )
    azimuth = np.mod(np.arctan2(y, x), 2 * np.pi)
    colatitude = np.arccos(np.clip(cos_colatitude, -1.0, 1.0))
    return np.where(nonzero, azimuth, 0.0), np.where(nonzero, colatitude, 0.0), radius


def sph2cart(azimuth, colatitude, radius):
    """Spherical to Cartesian coordinates."""
    x = radius * np.sin(colatitude) * np.cos(azimuth)
    y = radius * np.sin(colatitude) * np.sin(azimuth)
    z = radius * np.cos(colatitude)
    return x, y, z


def sh_index(degree: int, order: int) -> int:
    """Index of the real symmetric harmonic (degree, order), degree even."""
    return degree * (degree + 1) // 2 + order


def ishtmtx(azimuths, colatitudes, n_coefficients):
    """MRtrix-convention real symmetric SH matrix and its angular derivatives.

    Returns ``(Y, dY)`` with ``Y`` of shape (n, C) and ``dY`` of shape
    (2, n, C): ``dY[0]`` = d/dcolatitude, ``dY[1]`` = d/dazimuth
    (core.py:36-69).  Order
    m < 0 uses sqrt(2) Im(Y_l^|m|), m = 0 uses Re(Y_l^0), m > 0 uses
    sqrt(2) Re(Y_l^m), with SciPy's Condon-Shortley phase.
    """
    azimuths = np.atleast_1d(np.asarray(azimuths, dtype=np.float64))
    colatitudes = np.atleast_1d(np.asarray(colatitudes, dtype=np.float64))
    n = len(colatitudes)
    matrix = np.zeros((n_coefficients, n))
    derivative = np.zeros((n_coefficients, n, 2))
    degree, order = 0, 0
    for i in range(n_coefficients):
        m = abs(order)
        value, grad = scipy.special.sph_harm_y(degree, m, colatitudes, azimuths, diff_n=1)
        if order < 0:
            matrix[i] = np.sqrt(2) * np.imag(value)
            derivative[i] = np.sqrt(2) * np.imag(grad)
        elif order == 0:
            matrix[i] = np.real(value)
            derivative[i] = np.real(grad)
        else:
            matrix[i] = np.sqrt(2) * np.real(value)
            derivative[i] = np.sqrt(2) * np.real(grad)
        if degree == order:
            degree += 2
            order = -degree
        else:
            order += 1
    return matrix.T, derivative.T


def fibonacci_sphere(samples: int = 1000) -> np.ndarray:
    """Approximately uniform points on the unit sphere (Fibonacci lattice)."""
    phi = (1 + np.sqrt(5)) / 2
    golden_angle = 2 * np.pi / phi
    indices = np.arange(samples)
    theta = golden_angle * indices
    z = 1 - (2 * indices / (samples - 1))
    radius = np.sqrt(1 - z ** 2)
    return np.vstack((radius * np.cos(theta), radius * np.sin(theta), z)).T
