"""Utilities of the reference's public ``tractography.utils`` used by the path."""

from __future__ import annotations

import numpy as np


def normalize_odf(odf: np.ndarray) -> np.ndarray:
    """Scale every voxel's real SH coefficients to unit integral (utils.py:6-22):
    c / (sqrt(4 pi) c0) where c0 != 0, zero elsewhere."""
    normalized = np.zeros_like(odf)
    np.divide(odf / np.sqrt(4 * np.pi), odf[..., :1], out=normalized, where=odf[..., :1] != 0)
    return normalized
