"""Tracking domains (reference ``tractography/domain.py``).

``Image`` is the nonzero-voxel domain: a point is inside when its nearest
voxel, ``floor(A^-1 p + 0.5)`` (half-open cells ``[i - 0.5, i + 0.5)``), is
inside the image and nonzero (domain.py:358-382).  On the GPU the mask is a
``tg_domain`` of uint8 created once per runtime.

The reference also builds a voxel-face boundary mesh and a BVH in every
``Image`` constructor for boundary seeding and connectome end points
(domain.py:44-116, 219-264); the streamline tracker never reads them, so
this module does not build them.
"""

from __future__ import annotations

import ctypes
from abc import ABC, abstractmethod

import numpy as np

from . import _lib
from .nifti import apply_affine


class BaseDomain(ABC):
    """Region in which tracking continues (domain.py:20-216)."""

    @abstractmethod
    def contains(self, points) -> np.ndarray:
        """Authoritative membership test for (n, 3) world-space points."""


class Image(BaseDomain):
    """Domain of the nonzero voxels of a 3D image (domain.py:267-430)."""

    def __init__(self, image_data):
        if image_data.ndim != 3:
            raise ValueError("Only 3D images are supported for image domains.")
        self.values = np.ascontiguousarray(image_data.get_fdata() != 0, dtype=np.int32)
        self.dims = np.ascontiguousarray((*image_data.shape, 0), dtype=np.uint32)
        affine = image_data.affine
        self.affine = np.asarray(affine if affine is not None else np.eye(4), dtype=np.float64)
        self.inverse_affine = np.ascontiguousarray(np.linalg.inv(self.affine), dtype=np.float32)
        if not np.any(self.values):
            raise ValueError("Image domain must contain at least one nonzero voxel.")
        self._device = {}

    def contains(self, points) -> np.ndarray:
        """NumPy reference of domain.py:400-430."""
        voxel = np.floor(apply_affine(self.inverse_affine, points) + 0.5).astype(int)
        x, y, z = voxel[:, :3].T
        width, height, depth = self.values.shape
        inside = (0 <= x) & (x < width) & (0 <= y) & (y < height) & (0 <= z) & (z < depth)
        result = np.zeros(x.shape, dtype=np.bool_)
        result[inside] = self.values[x[inside], y[inside], z[inside]] != 0
        return result

    def device(self, runtime):
        """The ``tg_domain`` of this mask for ``runtime``."""
        key = id(runtime)
        obj = self._device.get(key)
        if obj is None:
            from .runtime import DeviceObject

            mask = np.ascontiguousarray(self.values != 0, dtype=np.uint8)
            nx, ny, nz = (int(v) for v in mask.shape)
            handle = ctypes.c_void_p()
            with runtime.device_scope():
                _lib.check(runtime.lib.tg_domain_create(
                    mask.ctypes.data_as(ctypes.c_void_p), nx, ny, nz,
                    self.inverse_affine.ctypes.data_as(ctypes.c_void_p),
                    ctypes.c_void_p(runtime.stream_handle), ctypes.byref(handle)))
            obj = DeviceObject(handle, runtime.lib.tg_domain_destroy)
            self._device[key] = obj
        return obj.handle


def contains(domain: BaseDomain, points, runtime=None) -> np.ndarray:
    """GPU membership test (domain.py:433-491)."""
    points = np.asarray(points)
    n = points.shape[0]
    if n == 0:
        return np.array([], dtype=np.bool_)
    if not isinstance(domain, Image):
        raise NotImplementedError(f"{type(domain).__name__} has no compiled CUDA code path")
    from .runtime import default_runtime

    runtime = runtime or default_runtime()
    import torch

    pts = np.zeros((n, 4), dtype=np.float32)
    pts[:, :3] = points
    pts[:, 3] = 1.0
    with runtime.device_scope():
        handle = domain.device(runtime)
        d_pts = runtime.to_device(pts)
        d_out = runtime.empty((n,), torch.uint8)
        _lib.check(runtime.lib.tg_domain_contains(handle, ctypes.c_void_p(d_pts.data_ptr()), n,
                                                  ctypes.c_void_p(d_out.data_ptr()),
                                                  ctypes.c_void_p(runtime.stream_handle)))
        return d_out.cpu().numpy().astype(bool)


def seed(domain: BaseDomain, n_seeds: int, rng_seed=None, runtime=None) -> np.ndarray:
    """Boundary seeding (domain.py:494-575) is not provided by this backend."""
    if not isinstance(n_seeds, (int, np.integer)) or n_seeds < 0:
        raise ValueError("n_seeds must be a non-negative integer.")
    if n_seeds == 0:
        return np.empty((0, 8), dtype=np.float32)
    raise NotImplementedError(
        "boundary seeding is not implemented by the CUDA backend; pass an (n_seeds, 8) seed array "
        "(for example from seeds.from_fod or seeds.from_mask)"
    )
