"""Seeded synthetic fields for the benchmark and the tests.

No public dataset is used.  The generators follow the workload definitions
of the benchmark configurations:

* ``config0``: 32^3 spherical-harmonic FOD (lmax 8, 45 coefficients), 2 mm
  isotropic voxels, generator seed 0.  Bundle A runs along x everywhere;
  bundle B follows circular arcs in the y-z plane (radius 10 voxels about
  the volume centre) inside a 4-voxel-thick torus.  Each fibre is a
  Watson-like zonal kernel exp(kappa (u.d)^2), kappa = 20, fitted by
  least squares on a dense Fibonacci grid (as the reference's test data is,
  test/data/__init__.py:104-110) and rotated to its direction; fractions are
  U[0.3, 0.7] normalised to one; N(0, 0.01) noise on every coefficient.
  Domain: ellipsoid mask with semi-axes 14/12/12 voxels.
* ``config1``: the same generator at 145 x 174 x 145 (1.25 mm) with three
  bundles: a slab along x, arcs in y-z, and a helix along z of pitch 40
  voxels.  Background voxels hold an isotropic FOD, so every voxel is
  nonzero and the default domain is the whole box.
* ``dti_field``: 6-coefficient tensors (1.7, 0.3, 0.3)e-3 mm^2/s along the
  config-0 directions with 5% log-normal eigenvalue jitter.

The SH basis is evaluated in float64 from the same exact polynomial tables
the CUDA kernels use (see csrc/gen_sh_tables.py), so generation needs no
SciPy and takes seconds even at the config-1 size.
"""

from __future__ import annotations

import numpy as np

from .csrc import gen_sh_tables as _tables
from .nifti import Nifti1Image

_KAPPA = 20.0


def _sh_tables_f64():
    """Per (l, m) exact-rounded-in-double polynomials of R_l^m."""
    from math import factorial, pi, sqrt

    out = []
    for l, m in _tables.pairs():
        exact = _tables.r_poly(l, m)
        k = sqrt((2 * l + 1) / (4 * pi) * factorial(l - m) / factorial(l + m)) * (sqrt(2.0) if m > 0 else 1.0)
        out.append((l, m, np.array([float(c) * k for c in exact[: l - m + 1]])))
    return out


_TABLE = None


def sh_basis(directions: np.ndarray, lmax: int = 8) -> np.ndarray:
    """Real symmetric SH basis (MRtrix order) at unit directions, float64 (n, C)."""
    global _TABLE
    if _TABLE is None:
        _TABLE = _sh_tables_f64()
    d = np.asarray(directions, dtype=np.float64)
    d = d / np.linalg.norm(d, axis=1, keepdims=True)
    x, y, z = d[:, 0], d[:, 1], d[:, 2]
    rho = np.hypot(x, y)
    st = rho
    ct = np.clip(z, -1.0, 1.0)
    with np.errstate(invalid="ignore", divide="ignore"):
        cp = np.where(rho > 0, x / np.where(rho > 0, rho, 1), 1.0)
        sp = np.where(rho > 0, y / np.where(rho > 0, rho, 1), 0.0)
    phi = np.arctan2(sp, cp)
    C = (lmax + 1) * (lmax + 2) // 2
    Y = np.zeros((len(d), C))
    for l, m, poly in _TABLE:
        if l > lmax:
            continue
        R = np.polynomial.polynomial.polyval(ct, poly)
        base = l * (l + 1) // 2
        if m == 0:
            Y[:, base] = R
        else:
            P = R * st ** m
            Y[:, base + m] = P * np.cos(m * phi)
            Y[:, base - m] = P * np.sin(m * phi)
    return Y


def fibonacci(n: int) -> np.ndarray:
    i = np.arange(n)
    golden_angle = 2 * np.pi / ((1 + np.sqrt(5)) / 2)
    z = 1 - 2 * i / (n - 1)
    r = np.sqrt(1 - z * z)
    return np.stack([r * np.cos(golden_angle * i), r * np.sin(golden_angle * i), z], axis=1)


def watson_zonal(lmax: int = 8, kappa: float = _KAPPA) -> np.ndarray:
    """Degree-l coefficients k_l (m = 0) of exp(kappa (u.z)^2), unit integral."""
    dirs = fibonacci(4000)
    Y = sh_basis(dirs, lmax)
    values = np.exp(kappa * (dirs[:, 2] ** 2 - 1.0))
    coef = np.linalg.lstsq(Y, values, rcond=None)[0]
    coef = coef / (coef[0] * np.sqrt(4 * np.pi))
    ks = {}
    for l in range(0, lmax + 1, 2):
        ks[l] = coef[l * (l + 1) // 2]
    return ks


def rotated_kernel(directions: np.ndarray, lmax: int = 8, kappa: float = _KAPPA) -> np.ndarray:
    """Coefficients of the zonal kernel rotated to each direction (n, C).

    Addition theorem: f(u.d) = sum_l k_l Y_l0(u) has coefficients
    c_lm = k_l sqrt(4 pi / (2l + 1)) Y_lm(d).
    """
    ks = watson_zonal(lmax, kappa)
    Y = sh_basis(directions, lmax)
    scale = np.zeros(Y.shape[1])
    for l in range(0, lmax + 1, 2):
        b = l * (l + 1) // 2
        scale[b - l: b + l + 1] = ks[l] * np.sqrt(4 * np.pi / (2 * l + 1))
    return Y * scale


def _mix(shape, bundles, rng, lmax, isotropic_background):
    """Sum of fibre kernels with U[0.3, 0.7] fractions normalised per voxel."""
    C = (lmax + 1) * (lmax + 2) // 2
    n = int(np.prod(shape))
    weights = np.zeros((n, len(bundles)))
    for b, (member, _) in enumerate(bundles):
        weights[member.ravel(), b] = rng.uniform(0.3, 0.7, size=int(member.sum()))
    total = weights.sum(axis=1)
    fod = np.zeros((n, C), dtype=np.float32)
    covered = total > 0
    weights[covered] /= total[covered, None]
    for b, (member, direction) in enumerate(bundles):
        idx = np.nonzero(member.ravel())[0]
        if np.ndim(direction) == 1:
            # one direction for the whole bundle: rotate the kernel once
            kernel = rotated_kernel(np.asarray(direction, float)[None, :], lmax)[0].astype(np.float32)
            fod[idx] += weights[idx, b, None].astype(np.float32) * kernel
            continue
        for start in range(0, len(idx), 262144):
            sel = idx[start: start + 262144]
            fod[sel] += (weights[sel, b, None] * rotated_kernel(direction.reshape(-1, 3)[sel], lmax)).astype(np.float32)
    if isotropic_background:
        fod[~covered, 0] = np.float32(1.0 / np.sqrt(4 * np.pi))
    return fod.reshape(*shape, C)


def config0(seed: int = 0, n: int = 32, voxel_mm: float = 2.0, lmax: int = 8):
    """Config-0 volume: (fod image, mask image)."""
    rng = np.random.default_rng(seed)
    c = (n - 1) / 2.0
    i, j, k = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    y, z = j - c, k - c
    r = np.hypot(y, z)
    dir_a = np.broadcast_to(np.array([1.0, 0.0, 0.0]), (n, n, n, 3))
    with np.errstate(invalid="ignore", divide="ignore"):
        dir_b = np.stack([np.zeros_like(r), -z / np.where(r > 0, r, 1), y / np.where(r > 0, r, 1)], axis=-1)
    torus = np.abs(r - 10.0) < 2.0
    bundles = [(np.ones((n, n, n), bool), dir_a), (torus, dir_b)]
    fod = _mix((n, n, n), bundles, rng, lmax, isotropic_background=False)
    fod += rng.normal(0.0, 0.01, size=fod.shape).astype(np.float32)
    affine = np.diag([voxel_mm, voxel_mm, voxel_mm, 1.0])
    mask = (((i - c) / 14.0) ** 2 + ((j - c) / 12.0) ** 2 + ((k - c) / 12.0) ** 2) <= 1.0
    return Nifti1Image(fod.astype(np.float32), affine), Nifti1Image(mask.astype(np.uint8), affine)


def config1(seed: int = 0, shape=(145, 174, 145), voxel_mm: float = 1.25, lmax: int = 8):
    """Config-1 volume (about 660 MB of float32): fod image."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    cx, cy, cz = (nx - 1) / 2.0, (ny - 1) / 2.0, (nz - 1) / 2.0
    i, j, k = np.meshgrid(np.arange(nx, dtype=np.float32), np.arange(ny, dtype=np.float32),
                          np.arange(nz, dtype=np.float32), indexing="ij")
    # bundle A: slab along x
    slab = np.abs(k - cz) < 20.0
    dir_a = np.broadcast_to(np.array([1.0, 0.0, 0.0], np.float32), shape + (3,))
    # bundle B: arcs in y-z about the centre, radius 40, thickness 10
    y, z = j - cy, k - cz
    r = np.hypot(y, z)
    arc = np.abs(r - 40.0) < 5.0
    with np.errstate(invalid="ignore", divide="ignore"):
        rr = np.where(r > 0, r, 1)
        dir_b = np.stack([np.zeros_like(r), -z / rr, y / rr], axis=-1)
    # bundle C: helix along z, pitch 40 voxels, radius 20, tube radius 6
    w = 2 * np.pi / 40.0
    hx, hy = cx + 20.0 * np.cos(w * k), cy + 20.0 * np.sin(w * k)
    helix = np.hypot(i - hx, j - hy) < 6.0
    tangent = np.stack([-20.0 * w * np.sin(w * k), 20.0 * w * np.cos(w * k), np.ones_like(k)], axis=-1)
    bundles = [(slab, dir_a), (arc, dir_b), (helix, tangent)]
    fod = _mix(shape, bundles, rng, lmax, isotropic_background=True)
    fod += rng.normal(0.0, 0.01, size=fod.shape).astype(np.float32)
    affine = np.diag([voxel_mm, voxel_mm, voxel_mm, 1.0])
    return Nifti1Image(fod, affine)


def bundle_field(shape, lmax: int = 8, seed: int = 0, voxel_mm: float = 2.0):
    """The config-0 generator at any grid size: bundle A along x everywhere and
    bundle B on circular arcs in y-z (radius 0.3 of the smaller y/z extent)
    inside a torus 4 voxels thick; fractions U[0.3, 0.7]; N(0, 0.01) noise.
    Returns (fod image, ellipsoid mask image with semi-axes 0.45 of each extent)."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    cy, cz = (ny - 1) / 2.0, (nz - 1) / 2.0
    i, j, k = np.meshgrid(np.arange(nx, dtype=np.float32), np.arange(ny, dtype=np.float32),
                          np.arange(nz, dtype=np.float32), indexing="ij")
    y, z = j - cy, k - cz
    r = np.hypot(y, z)
    radius = 0.3 * min(ny, nz)
    torus = np.abs(r - radius) < 2.0
    with np.errstate(invalid="ignore", divide="ignore"):
        rr = np.where(r > 0, r, 1)
        dir_b = np.stack([np.zeros_like(r), -z / rr, y / rr], axis=-1)
    bundles = [(np.ones(shape, bool), np.array([1.0, 0.0, 0.0])), (torus, dir_b)]
    fod = _mix(tuple(shape), bundles, rng, lmax, isotropic_background=False)
    fod += rng.normal(0.0, 0.01, size=fod.shape).astype(np.float32)
    affine = np.diag([voxel_mm, voxel_mm, voxel_mm, 1.0])
    cx = (nx - 1) / 2.0
    mask = (((i - cx) / (0.45 * nx)) ** 2 + ((j - cy) / (0.45 * ny)) ** 2 + ((k - cz) / (0.45 * nz)) ** 2) <= 1.0
    return Nifti1Image(fod.astype(np.float32), affine), Nifti1Image(mask.astype(np.uint8), affine)


MIXED_SHAPES = ((64, 64, 64), (96, 96, 60), (128, 128, 128), (145, 174, 145))


def mixed_job_specs(n_jobs: int = 64, seed: int = 0, max_seeds: int = 500_000, min_seeds: int = 1000):
    """Config-3 job draws: volume size, lmax (4/6/8), seed count log-U[1k, 500k],
    Transport or Diffusion (noise variance U[0.05, 0.2]), maximum length U[50, 300] mm."""
    rng = np.random.default_rng(seed)
    specs = []
    for _ in range(n_jobs):
        specs.append({
            "shape": MIXED_SHAPES[int(rng.integers(0, len(MIXED_SHAPES)))],
            "lmax": int(rng.choice([4, 6, 8])),
            "n_seeds": int(np.exp(rng.uniform(np.log(min_seeds), np.log(max_seeds)))),
            "algorithm": "transport" if rng.uniform() < 0.5 else "diffusion",
            "noise_variance": float(rng.uniform(0.05, 0.2)),
            "max_length": float(rng.uniform(50.0, 300.0)),
            "seed": int(rng.integers(0, 2 ** 31)),
        })
    return specs


def uniform_seeds(mask_img, n: int, seed: int = 0) -> np.ndarray:
    """n seeds uniform in the mask's nonzero voxels with uniform orientations."""
    rng = np.random.default_rng(seed)
    vox = np.argwhere(np.asarray(mask_img.dataobj) != 0)
    pick = vox[rng.integers(0, len(vox), n)] + rng.uniform(-0.5, 0.5, (n, 3))
    loc = pick @ np.asarray(mask_img.affine)[:3, :3].T + np.asarray(mask_img.affine)[:3, 3]
    o = rng.normal(size=(n, 3))
    o /= np.linalg.norm(o, axis=1, keepdims=True)
    out = np.empty((n, 8), np.float32)
    out[:, :3], out[:, 3], out[:, 4:7], out[:, 7] = loc, 1.0, o, 0.0
    return out


def dti_field(shape=(96, 96, 60), seed: int = 0, voxel_mm: float = 2.0):
    """6-coefficient tensors along the config-0 directions with 5% log-normal jitter."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    cy, cz = (ny - 1) / 2.0, (nz - 1) / 2.0
    i, j, k = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    y, z = j - cy, k - cz
    r = np.hypot(y, z)
    torus = np.abs(r - min(cy, cz) * 0.6) < 2.0
    with np.errstate(invalid="ignore", divide="ignore"):
        rr = np.where(r > 0, r, 1)
        d = np.where(torus[..., None], np.stack([np.zeros_like(r), -z / rr, y / rr], -1),
                     np.array([1.0, 0.0, 0.0]))
    d = d / np.linalg.norm(d, axis=-1, keepdims=True)
    ev = np.array([1.7e-3, 0.3e-3, 0.3e-3]) * np.exp(rng.normal(0, 0.05, size=shape + (3,)))
    # orthonormal frame (d, e1, e2)
    helper = np.where(np.abs(d[..., :1]) < 0.9, np.array([1.0, 0, 0]), np.array([0, 1.0, 0]))
    e1 = np.cross(d, helper)
    e1 /= np.linalg.norm(e1, axis=-1, keepdims=True)
    e2 = np.cross(d, e1)
    D = (ev[..., 0, None, None] * d[..., :, None] * d[..., None, :]
         + ev[..., 1, None, None] * e1[..., :, None] * e1[..., None, :]
         + ev[..., 2, None, None] * e2[..., :, None] * e2[..., None, :])
    coeffs = np.stack([D[..., 0, 0], D[..., 1, 1], D[..., 2, 2], D[..., 0, 1], D[..., 0, 2], D[..., 1, 2]], -1)
    affine = np.diag([voxel_mm, voxel_mm, voxel_mm, 1.0])
    return Nifti1Image(coeffs.astype(np.float32), affine)


def seeds_in_mask(mask_img, n: int, seed: int = 0) -> np.ndarray:
    """``seeds.from_mask`` semantics with a fixed NumPy legacy seed."""
    from . import seeds as seeds_module

    state = np.random.get_state()
    np.random.seed(seed)
    try:
        return seeds_module.from_mask(mask_img, n)
    finally:
        np.random.set_state(state)


def geodesic_sphere(frequency: int):
    """Unit geodesic sphere: each icosahedron face cut into frequency^2
    triangles, points projected to the sphere.  Shared edge and corner
    points are generated once, so the surface is closed; faces are wound
    outward.  Returns (vertices (V, 3) float64, faces (20 f^2, 3) uint32)."""
    n = int(frequency)
    if n < 1:
        raise ValueError("frequency must be >= 1")
    t = (1.0 + 5.0 ** 0.5) / 2.0
    corners = np.array([[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t],
                        [0, -1, -t], [0, 1, -t], [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    ico = np.array([[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4],
                    [11, 10, 2], [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
                    [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]])
    points = [c for c in corners]
    index = {("c", k): k for k in range(12)}

    def vertex(key, position):
        k = index.get(key)
        if k is None:
            k = len(points)
            index[key] = k
            points.append(position)
        return k

    def edge_point(a, b, k):
        if k == 0:
            return a
        if k == n:
            return b
        if a > b:
            a, b, k = b, a, n - k
        return vertex(("e", a, b, k), corners[a] + (corners[b] - corners[a]) * (k / n))

    faces = []
    for f, (A, B, C) in enumerate(ico):
        grid = {}
        for i in range(n + 1):
            for j in range(n + 1 - i):
                if j == 0:
                    grid[i, j] = edge_point(A, B, i)
                elif i == 0:
                    grid[i, j] = edge_point(A, C, j)
                elif i + j == n:
                    grid[i, j] = edge_point(B, C, j)
                else:
                    p = corners[A] + (corners[B] - corners[A]) * (i / n) + (corners[C] - corners[A]) * (j / n)
                    grid[i, j] = vertex(("f", f, i, j), p)
        for i in range(n):
            for j in range(n - i):
                faces.append((grid[i, j], grid[i + 1, j], grid[i, j + 1]))
                if i + j < n - 1:
                    faces.append((grid[i + 1, j], grid[i + 1, j + 1], grid[i, j + 1]))
    v = np.asarray(points, dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    faces = np.asarray(faces, dtype=np.int64)
    tri = v[faces]
    normal = np.cross(tri[:, 1] - tri[:, 0], tri[:, 2] - tri[:, 0])
    inward = np.einsum("ij,ij->i", normal, tri.mean(axis=1)) < 0
    faces[inward] = faces[inward][:, [0, 2, 1]]
    return v, faces.astype(np.uint32)


def config2_surface(shape=(96, 96, 60), voxel_mm: float = 2.0, frequency: int = 158, fill: float = 0.9):
    """Closed surface of the DTI/mesh workload: a geodesic sphere (20 f^2
    triangles; f = 158 gives 499 280) with radius r = 1 + 0.1 Y_2^1 + 0.05 Y_4^0
    (real orthonormal harmonics), scaled per axis so that its extent is
    `fill` of the volume's and centred in it (world mm, affine diag(voxel))."""
    v, f = geodesic_sphere(frequency)
    x, y, z = v.T
    ct = np.clip(z, -1.0, 1.0)
    st = np.sqrt(np.maximum(0.0, 1.0 - ct * ct))
    phi = np.arctan2(y, x)
    y21 = np.sqrt(15.0 / (4.0 * np.pi)) * st * ct * np.cos(phi)
    y40 = 3.0 / 16.0 * np.sqrt(1.0 / np.pi) * (35.0 * ct ** 4 - 30.0 * ct ** 2 + 3.0)
    r = 1.0 + 0.1 * y21 + 0.05 * y40
    v = v * r[:, None]
    lo, hi = v.min(axis=0), v.max(axis=0)
    extent = (np.asarray(shape, dtype=np.float64) - 1.0) * voxel_mm
    scale = fill * extent / (hi - lo)
    centre = extent / 2.0
    v = (v - (lo + hi) / 2.0) * scale + centre
    return v, f


def seeds_inside(contains, bounds_lo, bounds_hi, n: int, seed: int = 0, chunk: int = 1 << 20) -> np.ndarray:
    """n seeds uniform inside a region given by a vectorised ``contains``
    over its bounding box (rejection sampling), with uniform orientations."""
    rng = np.random.default_rng(seed)
    lo, hi = np.asarray(bounds_lo, np.float64), np.asarray(bounds_hi, np.float64)
    kept = []
    have = 0
    while have < n:
        p = rng.uniform(lo, hi, (chunk, 3))
        p = p[np.asarray(contains(p), dtype=bool)]
        kept.append(p)
        have += len(p)
    loc = np.concatenate(kept)[:n]
    o = rng.normal(size=(n, 3))
    o /= np.linalg.norm(o, axis=1, keepdims=True)
    out = np.empty((n, 8), np.float32)
    out[:, :3], out[:, 3], out[:, 4:7], out[:, 7] = loc, 1.0, o, 0.0
    return out


def config1_workload(n_seeds: int, runtime, *, numpy_seed: int = 2024, algorithm_seed: int = 1234):
    """The single-volume Diffusion job: the 145x174x145 lmax-8 volume of
    ``config1(seed=0)``, its nonzero voxels as the domain, ``n_seeds`` seeds
    from ``seeds.from_fod`` under ``numpy.random.seed(numpy_seed)`` (the
    global RNG is restored afterwards), and Diffusion with step 0.001 mm,
    gamma 1, noise variance 0.1 seeded by ``algorithm_seed``.

    Returns (fod image, field, domain, seeds, algorithm)."""
    from . import algorithm as _algorithm
    from . import domain as _domain
    from . import field as _field
    from . import local as _local
    from . import seeds as _seeds

    fod = config1(seed=0)
    field = _field.Image(fod)
    mask = np.any(field.values != 0, axis=-1).astype(np.uint8)
    domain = _domain.Image(Nifti1Image(mask, fod.affine))
    state = np.random.get_state()
    np.random.seed(numpy_seed)
    try:
        seeds = _seeds.from_fod(fod, n_seeds, runtime=runtime)
    finally:
        np.random.set_state(state)
    model = _local.RealSymmetricSphericalHarmonics(45)
    algorithm = _algorithm.Diffusion(model, step_size=0.001, gamma=1.0, noise_variance=0.1, seed=algorithm_seed)
    return fod, field, domain, seeds, algorithm


def config2_workload(n_seeds: int, runtime, *, step_size: float = 0.2):
    """The tensor job in a closed-surface domain: 96x96x60 tensors at 2 mm
    (``dti_field(seed=0)``), the ~499k-triangle surface of
    ``config2_surface()``, ``n_seeds`` seeds uniform inside it (seed 5) and
    Transport at 0.1 voxel.

    Returns (field, mesh domain, seeds, algorithm)."""
    from . import algorithm as _algorithm
    from . import domain as _domain
    from . import field as _field
    from . import local as _local

    fod = dti_field(shape=(96, 96, 60), seed=0)
    field = _field.Image(fod)
    v, f = config2_surface()
    mesh = _domain.Mesh(v, f)
    seeds = seeds_inside(lambda p: _domain.contains(mesh, p, runtime), v.min(axis=0), v.max(axis=0), n_seeds,
                         seed=5)
    algorithm = _algorithm.Transport(_local.DiffusionTensorImaging(), step_size=step_size, gamma=1.0)
    return field, mesh, seeds, algorithm
