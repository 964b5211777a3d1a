"""Image container used by the public API.

The reference takes ``nibabel.nifti1.Nifti1Image`` objects.  When nibabel is
installed its class is used as is; otherwise this module provides a minimal
in-memory stand-in with the attributes the tracker reads (``dataobj``,
``affine``, ``shape``, ``ndim``, ``get_fdata``).  File I/O of NIfTI is out
of scope for the tracking path.
"""

from __future__ import annotations

import numpy as np

try:  # pragma: no cover - depends on the environment
    from nibabel.nifti1 import Nifti1Image as _NibabelImage
except ImportError:  # pragma: no cover
    _NibabelImage = None


class _ArrayImage:
    """In-memory image with an affine (subset of nibabel's SpatialImage)."""

    def __init__(self, dataobj, affine=None, header=None):
        self._data = np.asanyarray(dataobj)
        self.affine = None if affine is None else np.asarray(affine, dtype=np.float64)
        self.header = header

    @property
    def dataobj(self):
        return self._data

    @property
    def shape(self):
        return self._data.shape

    @property
    def ndim(self):
        return self._data.ndim

    def get_fdata(self, dtype=np.float64):
        return np.asarray(self._data, dtype=dtype)


Nifti1Image = _NibabelImage if _NibabelImage is not None else _ArrayImage


def is_image(obj) -> bool:
    """True for a nibabel image or the in-memory stand-in."""
    if isinstance(obj, _ArrayImage):
        return True
    return _NibabelImage is not None and isinstance(obj, _NibabelImage)


def apply_affine(affine, points):
    """``nibabel.affines.apply_affine`` for (n, 3) points."""
    affine = np.asarray(affine)
    points = np.asarray(points)
    return points @ affine[:3, :3].T + affine[:3, 3]
