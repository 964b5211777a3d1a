"""Seed generation (reference ``tractography/seeds.py``).

Seeds are (n, 8) float32 rows ``(x, y, z, 1, dx, dy, dz, 0)``.
``from_fod`` importance-samples an orientation per seed from the local FOD
over 1000 Fibonacci directions on the GPU (seeds.cl:68-118); its per-seed
MWC64X states are drawn from NumPy's legacy global generator exactly as the
reference does (seeds.py:185), so ``np.random.seed`` makes it reproducible.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

from . import _lib
from . import core
from . import local as local_models
from .nifti import apply_affine


def _from_components(locations, orientations) -> np.ndarray:
    """Canonical (n, 8) homogeneous seed array (seeds.py:16-32)."""
    locations = np.asarray(locations, dtype=np.float32)
    orientations = np.asarray(orientations, dtype=np.float32)
    if locations.ndim != 2 or locations.shape[1] != 3:
        raise ValueError("locations must have shape (n_seeds, 3).")
    if orientations.shape != locations.shape:
        raise ValueError("orientations must have the same shape as locations.")
    result = np.empty((len(locations), 8), dtype=np.float32)
    result[:, :3] = locations
    result[:, 3] = 1.0
    result[:, 4:7] = orientations
    result[:, 7] = 0.0
    return result


def validate_seed_array(seeds) -> np.ndarray:
    """Validate a canonical seed array (seeds.py:35-54)."""
    result = np.ascontiguousarray(seeds, dtype=np.float32)
    if result.ndim != 2 or result.shape[1] != 8:
        raise ValueError("seeds must have shape (n_seeds, 8).")
    if not np.all(result[:, 3] == 1) or not np.all(result[:, 7] == 0):
        raise ValueError("seed position and orientation homogeneous values must be 1 and 0.")
    return result


def from_surface(surface, n_seeds: int, cone_angle: float = 0):
    """Surface seeding needs the nimesh package, which this backend does not use."""
    if n_seeds == 0:
        return np.empty((0, 8), dtype=np.float32)
    raise NotImplementedError("from_surface is not provided by the CUDA backend")


def from_mask(mask, n_seeds: int) -> np.ndarray:
    """Uniform seeds in nonzero voxels, uniform orientations (seeds.py:114-142)."""
    if n_seeds == 0:
        return np.empty((0, 8), dtype=np.float32)
    voxels = np.array(list(zip(*np.nonzero(mask.get_fdata()))))
    indices = np.random.randint(len(voxels), size=n_seeds)
    locations_voxel = voxels[indices] + np.random.rand(n_seeds, 3) - [0.5, 0.5, 0.5]
    locations = apply_affine(mask.affine, locations_voxel)
    orientations = np.random.randn(n_seeds, 3)
    orientations /= np.linalg.norm(orientations, axis=1, keepdims=True)
    return _from_components(locations, orientations)


def sparse_fod(fod):
    """Nonzero voxels of a 4D FOD image: (coefficients, voxel indices with w=1, affine)."""
    data = fod.get_fdata()
    mask = np.any(data != 0, axis=-1)
    indices = np.array(np.nonzero(mask), dtype=np.float32).T
    voxels = np.hstack((indices, np.ones((len(indices), 1)))).astype(np.float32)
    inline_fod = data[mask].astype(np.float32)
    affine = np.asarray(fod.affine).astype(np.float32)
    return inline_fod, voxels, affine


def from_fod(fod, n_seeds: int, use_opencl: bool = True, *, runtime=None) -> np.ndarray:
    """Seeds uniform in nonzero FOD voxels, orientations sampled from the FOD.

    ``use_opencl`` keeps the reference's keyword: True runs the GPU kernel,
    False the NumPy path (seeds.py:218-240).
    """
    if n_seeds == 0:
        return np.empty((0, 8), dtype=np.float32)
    if not use_opencl:
        data = fod.get_fdata()
        voxels = np.array(list(zip(*np.nonzero(np.any(data != 0, axis=-1)))))
        indices = np.random.randint(len(voxels), size=n_seeds)
        locations_voxel = voxels[indices] + np.random.rand(n_seeds, 3) - [0.5, 0.5, 0.5]
        locations = apply_affine(fod.affine, locations_voxel)
        vertices = core.fibonacci_sphere(1000)
        az, co, _ = core.cart2sph(*vertices.T)
        mtx, _ = core.ishtmtx(az, co, fod.shape[-1])
        orientations = []
        for index in indices:
            values = np.dot(mtx, data[tuple(voxels[index])])
            cumsum = np.cumsum(np.maximum(values, 0.0))
            i = np.searchsorted(cumsum, np.random.rand() * cumsum[-1])
            orientations.append(vertices[i])
        return _from_components(locations, orientations)

    from .runtime import default_runtime

    runtime = runtime or default_runtime()
    inline_fod, voxels, affine = sparse_fod(fod)
    randoms = np.random.randint(4294967295, size=(n_seeds, 2)).astype(np.uint32)
    model = local_models.from_shape(fod.shape)
    return seeds_from_sparse_fod(model.model_id, inline_fod, voxels, affine, randoms, runtime)


def seeds_from_sparse_fod(model: int, inline_fod, voxels, affine, states, runtime) -> np.ndarray:
    """Run the FOD seeding kernel on prepared sparse inputs."""
    import torch

    n = int(states.shape[0])
    with runtime.device_scope():
        d_fod = runtime.to_device(np.ascontiguousarray(inline_fod, dtype=np.float32))
        d_vox = runtime.to_device(np.ascontiguousarray(voxels, dtype=np.float32))
        d_aff = runtime.to_device(np.ascontiguousarray(affine, dtype=np.float32))
        d_states = runtime.to_device(np.ascontiguousarray(states, dtype=np.uint32).view(np.int32))
        d_out = runtime.empty((n, 8), torch.float32)
        _lib.check(runtime.lib.tg_seeds_from_fod(
            model, int(inline_fod.shape[1]), ctypes.c_void_p(d_fod.data_ptr()), ctypes.c_void_p(d_vox.data_ptr()),
            int(voxels.shape[0]), ctypes.c_void_p(d_aff.data_ptr()), ctypes.c_void_p(d_states.data_ptr()), n,
            ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(runtime.stream_handle)))
        return d_out.cpu().numpy()


def save(filename: Path, seeds) -> None:
    """Save seeds as .txt (six columns) or .tck (two-point streamlines) (seeds.py:243-270)."""
    from .streamlines import Tractogram, save_tck

    seeds = validate_seed_array(seeds)
    filename = Path(filename)
    match filename.suffix:
        case ".txt":
            np.savetxt(filename, np.hstack((seeds[:, :3], seeds[:, 4:7])))
        case ".tck":
            data = [np.vstack((s[:3], s[:3] + s[4:7])) for s in seeds]
            save_tck(filename, Tractogram(data, affine_to_rasmm=np.eye(4)))
        case _:
            raise ValueError(f"Unknown file type {filename.suffix}")


def load(filename: Path) -> np.ndarray:
    """Load seeds saved by :func:`save` (seeds.py:273-303)."""
    from .streamlines import load_tck

    filename = Path(filename)
    match filename.suffix:
        case ".txt":
            data = np.loadtxt(filename, dtype=np.float32, ndmin=2)
            if data.size == 0:
                return np.empty((0, 8), dtype=np.float32)
            if data.shape[1] != 6:
                raise ValueError("Text seed files must contain six columns.")
            return _from_components(data[:, :3], data[:, 3:6])
        case ".tck":
            streamlines = load_tck(filename).streamlines
            locations = np.asarray([s[0] for s in streamlines], dtype=np.float32).reshape(-1, 3)
            orientations = np.asarray([s[1] - s[0] for s in streamlines], dtype=np.float32).reshape(-1, 3)
            return _from_components(locations, orientations)
        case _:
            raise ValueError(f"Unknown file type {filename.suffix}")
