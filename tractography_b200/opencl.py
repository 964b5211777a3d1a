"""Compatibility names for code written against ``tractography.opencl``.

The reference exposes ``OpenCLRuntime`` and ``BufferAccess``
(``tractography/opencl.py:22-163``) and its public functions take a
``runtime=`` argument.  Here the runtime is :class:`CudaRuntime`; the old
names remain importable so callers do not have to change.  There is no
OpenCL backend and no CPU fallback.
"""

from enum import Enum

from .runtime import CudaRuntime


class BufferAccess(Enum):
    """Kernel-side access mode of a buffer (kept for API compatibility)."""

    READ_ONLY = 1
    WRITE_ONLY = 2
    READ_WRITE = 4


OpenCLRuntime = CudaRuntime

__all__ = ["BufferAccess", "CudaRuntime", "OpenCLRuntime"]
