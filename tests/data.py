"""Synthetic fields used by the tests.

Same definitions as the reference's test fixtures (test/data/__init__.py,
test/data/tensor.py): tensor-shaped ODFs exp(-u^T D u) sampled on a
Fibonacci grid and fitted to real symmetric SH by least squares, then
normalised to unit integral; DTI fields hold the six tensor coefficients.
"""

from __future__ import annotations

import numpy as np

import tractography_b200 as tg

_BALL = np.diag([5.0, 5.0, 5.0])
_X_TENSOR = np.diag([5.0, 1.0, 5.0])
_Y_TENSOR = np.diag([1.0, 5.0, 5.0])


def normalize_odf(odf):
    """Scale each voxel's SH coefficients to unit integral (c0 = 1/sqrt(4 pi))."""
    out = np.zeros_like(odf)
    np.divide(odf / np.sqrt(4 * np.pi), odf[..., :1], out=out, where=odf[..., :1] != 0)
    return out


def _fit(values, bvectors, n_coefficients):
    az, co, _ = tg.core.cart2sph(*bvectors.T)
    Y, _ = tg.core.ishtmtx(az, co, n_coefficients)
    return normalize_odf(np.tensordot(values, np.linalg.pinv(Y), axes=(3, 1)))


def _tensor_odf(tensor, shape, bvectors):
    field = np.zeros(shape + (len(bvectors),))
    field[..., :] = np.exp(-np.einsum("ni,ij,nj->n", bvectors, tensor, bvectors))
    return field


def uniform_isotropic(shape=(10, 10, 10), n_coefficients=45):
    b = tg.core.fibonacci_sphere(n_coefficients * 3)
    return _fit(_tensor_odf(_BALL, shape, b), b, n_coefficients)


def circle(shape=(10, 10, 1), n_coefficients=45, radius=2, width=1):
    b = tg.core.fibonacci_sphere(n_coefficients * 3)
    values = np.zeros(shape + (len(b),))
    center = np.array(shape, dtype=float) / 2 - 0.5
    for i, j, k in np.ndindex(*shape):
        x, y, _ = np.r_[i, j, k] - center
        r = np.hypot(x, y)
        if radius - width < r < radius + width:
            frame = np.array([[y / r, x / r, 0], [-x / r, y / r, 0], [0, 0, 1.0]])
            tensor = frame @ np.diag([1.0, 5.0, 5.0]) @ frame.T
            values[i, j, k] = np.exp(-np.einsum("ni,ij,nj->n", b, tensor, b))
    return _fit(values, b, n_coefficients)


def cross(shape=(10, 10, 1), n_coefficients=45):
    b = tg.core.fibonacci_sphere(n_coefficients * 3)
    values = _tensor_odf(_BALL, shape, b)
    xo = shape[0] // 3
    values[xo:-xo] = _tensor_odf(_X_TENSOR, (shape[0] - 2 * xo, shape[1], shape[2]), b)
    yo = shape[1] // 3
    values[:, yo:-yo] += _tensor_odf(_Y_TENSOR, (shape[0], shape[1] - 2 * yo, shape[2]), b)
    fod = tg.Nifti1Image(_fit(values, b, n_coefficients), np.eye(4))
    mask = np.zeros(shape, dtype=np.uint8)
    mask[xo:-xo] = 1
    mask[:, yo:-yo] = 1
    return fod, tg.Nifti1Image(mask, np.eye(4))


def cross_segmentation(shape=(10, 10, 1)):
    """Regions 1-4 at the four ends of the cross (test/data/__init__.py:86-92)."""
    xo, yo = shape[0] // 3, shape[1] // 3
    seg = np.zeros(shape, dtype=np.uint8)
    seg[xo:-xo, 0] = 1
    seg[xo:-xo, -1] = 2
    seg[0, yo:-yo] = 3
    seg[-1, yo:-yo] = 4
    return tg.Nifti1Image(seg, np.eye(4))


def tensor_circle(shape=(20, 20, 1), radius=5, width=2):
    values = np.zeros(shape + (6,))
    values[..., :3] = 0.003
    wm = np.zeros(shape, dtype=np.uint8)
    center = np.array(shape, dtype=float) / 2 - 0.5
    affine = np.eye(4)
    affine[:3, 3] = center
    for i, j, k in np.ndindex(*shape):
        x, y, _ = np.r_[i, j, k] - center
        r = np.hypot(x, y)
        if radius - width < r < radius + width:
            frame = np.array([[y / r, x / r, 0], [-x / r, y / r, 0], [0, 0, 1.0]])
            tensor = frame @ (np.diag([1.5, 0.4, 0.4]) / 1000) @ frame.T
            values[i, j, k] = tensor[[0, 1, 2, 0, 0, 1], [0, 1, 2, 1, 2, 2]]
            wm[i, j, k] = 1
    return tg.Nifti1Image(values, affine), tg.Nifti1Image(wm, affine)


def tensor_cross(shape=(20, 20, 1)):
    values = np.zeros(shape + (6,))
    wm = np.zeros(shape, dtype=np.uint8)
    values[..., :3] = 0.003
    xo, yo = shape[0] // 3, shape[1] // 3
    xs, ys = shape[0] - 2 * xo, shape[1] - 2 * yo
    values[xo:xo + xs, :, :, :3] = 0
    values[:, yo:yo + ys, :, :3] = 0
    center = np.array(shape, dtype=float) / 2 - 0.5
    affine = np.eye(4)
    affine[:3, 3] = center
    values[xo:xo + xs, :, :, :3] += [0.4e-3, 1.5e-3, 0.4e-3]
    wm[xo:xo + xs] = 1
    values[:, yo:yo + ys, :, :3] += [1.5e-3, 0.4e-3, 0.4e-3]
    wm[:, yo:yo + ys] = 1
    return tg.Nifti1Image(values, affine), tg.Nifti1Image(wm, affine)


def u0u3_coefficients(epsilon=0.3, n_coefficients=45):
    """SH fit of F(u) = 1 + epsilon u_x u_z (test_algorithms/exact_solutions.py:6-12)."""
    d = tg.core.fibonacci_sphere(5000)
    az, co, _ = tg.core.cart2sph(*d.T)
    Y, _ = tg.core.ishtmtx(az, co, n_coefficients)
    return np.linalg.pinv(Y) @ (1.0 + epsilon * d[:, 0] * d[:, 2])


def u0u3_reference(step_size, gamma, theta_0, phi_0, epsilon, n_steps):
    """Forward-Euler orientations of the analytic u0u3 drift (exact_solutions.py:15-37)."""
    u = np.asarray(tg.core.sph2cart(phi_0, theta_0, 1.0), dtype=float)
    out = [u.copy()]
    for _ in range(n_steps - 1):
        value = 1.0 + epsilon * u[0] * u[2]
        grad = np.array([u[2], 0.0, u[0]])
        tangent = (np.eye(3) - np.outer(u, u)) @ grad * gamma * epsilon / value
        u = u + step_size * tangent
        u /= np.linalg.norm(u)
        out.append(u.copy())
    return np.asarray(out)
