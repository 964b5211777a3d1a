"""Fields of local-model parameters (reference ``tractography/field.py``).

``Image`` holds a 4D float32 coefficient image sampled at the nearest voxel
with ties-to-even rounding (field.py:88-114).  On the GPU the image lives
once per runtime as a ``tg_field`` (voxel-major, coefficients padded to a
multiple of four floats); the reference re-uploaded it for every batch.
"""

from __future__ import annotations

import ctypes
from abc import ABC, abstractmethod

import numpy as np

from . import _lib
from .nifti import apply_affine


class BaseField(ABC):
    """A field of local-model parameters (field.py:15-49)."""

    def __init__(self, n_parameters: int):
        self.n_parameters = n_parameters

    @abstractmethod
    def evaluate(self, points):
        """Evaluate the field at world-space points (NumPy reference)."""


class Image(BaseField):
    """Nearest-neighbour image field (field.py:52-141)."""

    def __init__(self, image_data):
        if image_data.ndim != 4:
            raise ValueError("Only 4D images are supported for image fields.")
        super().__init__(image_data.shape[3])
        self.values = np.ascontiguousarray(image_data.get_fdata(), dtype=np.float32)
        self.dims = np.ascontiguousarray(image_data.shape, dtype=np.uint32)
        affine = image_data.affine
        self.inverse_affine = np.ascontiguousarray(
            np.linalg.inv(affine if affine is not None else np.eye(4)), dtype=np.float32
        )
        self._device = {}

    def evaluate(self, points):
        """NumPy reference: rint(A^-1 p), zero outside the image."""
        voxel = np.round(apply_affine(self.inverse_affine, points)).astype(int)
        x, y, z = voxel[:, :3].T
        width, height, depth, n_parameters = self.values.shape
        inside = (0 <= x) & (x < width) & (0 <= y) & (y < height) & (0 <= z) & (z < depth)
        result = np.zeros((points.shape[0], n_parameters), dtype=np.float32)
        result[inside, :] = self.values[x[inside], y[inside], z[inside]]
        return result

    def device(self, runtime, model: int):
        """The ``tg_field`` of this image for ``runtime`` and model id."""
        key = (id(runtime), model)
        obj = self._device.get(key)
        if obj is None:
            from .runtime import DeviceObject

            handle = ctypes.c_void_p()
            nx, ny, nz, nc = (int(v) for v in self.values.shape)
            with runtime.device_scope():
                _lib.check(runtime.lib.tg_field_create(
                    model, self.values.ctypes.data_as(ctypes.c_void_p), nx, ny, nz, nc,
                    self.inverse_affine.ctypes.data_as(ctypes.c_void_p),
                    ctypes.c_void_p(runtime.stream_handle), ctypes.byref(handle)))
            obj = DeviceObject(handle, runtime.lib.tg_field_destroy)
            self._device[key] = obj
        return obj.handle


def evaluate(field: BaseField, points, runtime=None) -> np.ndarray:
    """Evaluate ``field`` at (n, 3) points on the GPU (field.py:144-197)."""
    points = np.asarray(points)
    n = points.shape[0]
    if n == 0:
        return np.empty((0, field.n_parameters), dtype=np.float32)
    if not isinstance(field, Image):
        raise NotImplementedError(f"{type(field).__name__} has no compiled CUDA code path")
    from .runtime import default_runtime

    runtime = runtime or default_runtime()
    import torch

    pts = np.zeros((n, 4), dtype=np.float32)
    pts[:, :3] = points
    pts[:, 3] = 1.0
    with runtime.device_scope():
        handle = field.device(runtime, _lib.MODEL_SH if field.n_parameters <= 45 else -1)
        d_pts = runtime.to_device(pts)
        d_out = runtime.empty((n, field.n_parameters), torch.float32)
        _lib.check(runtime.lib.tg_field_evaluate(handle, ctypes.c_void_p(d_pts.data_ptr()), n,
                                                 ctypes.c_void_p(d_out.data_ptr()),
                                                 ctypes.c_void_p(runtime.stream_handle)))
        return d_out.cpu().numpy()
