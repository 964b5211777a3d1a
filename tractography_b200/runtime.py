"""CUDA runtime for the tracker: device, stream and the library objects.

Replaces ``OpenCLRuntime`` (reference ``tractography/opencl.py:30-163``),
which owned an OpenCL context and queue and compiled a program for every
call.  Here the kernels are compiled ahead of time into ``libtg_b200.so``;
the runtime owns the CUDA stream the calls are ordered on and one
persistent tracker (its point pool and per-seed buffers are reused across
calls).  PyTorch provides device selection, streams and pinned host memory.
"""

from __future__ import annotations

import ctypes
import weakref

import numpy as np

from . import _lib


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError(
            "tractography_b200 requires a CUDA device (B200, sm_100a); none is available"
        )
    return torch


class CudaRuntime:
    """Own the CUDA device and stream used for tracking.

    Args:
        device: CUDA device index or ``torch.device``; defaults to the current
            device.
        stream: ``torch.cuda.Stream`` to order work on; defaults to the
            device's current stream.
        pool_points: capacity of the tracker's point pool (0 sizes it on
            first use from the free device memory).
    """

    def __init__(self, device=None, *, stream=None, pool_points: int = 0):
        torch = _torch()
        if device is None:
            device = torch.cuda.current_device()
        self.device = torch.device("cuda", device if isinstance(device, int) else torch.device(device).index)
        self.stream = stream if stream is not None else torch.cuda.current_stream(self.device)
        self.lib = _lib.load()
        self.pool_points = int(pool_points)
        self._tracker = None
        self._finalizer = None

    @property
    def stream_handle(self) -> int:
        return int(self.stream.cuda_stream)

    @property
    def queue(self):
        """The stream, under the attribute name the OpenCL runtime used."""
        return self.stream

    def tracker(self) -> ctypes.c_void_p:
        if self._tracker is None:
            handle = ctypes.c_void_p()
            with self.device_scope():
                _lib.check(self.lib.tg_tracker_create(self.pool_points, ctypes.byref(handle)))
            self._tracker = handle
            self._finalizer = weakref.finalize(self, _destroy, self.lib.tg_tracker_destroy, handle)
        return self._tracker

    def set_tuning(self, blocks_per_sm: int = 0, compact_lanes: int = 0, compact_rounds: int = 4) -> None:
        """Launch shape and tail compaction of the tracker (results do not depend on them)."""
        _lib.check(self.lib.tg_tracker_set_tuning(self.tracker(), blocks_per_sm, compact_lanes, compact_rounds))

    def set_slicing(self, slice_steps: int) -> None:
        """Time slicing of the tracker's persistent launch: 0 (off) or a power
        of two, the steps after which a streamline yields its lane while other
        work waits (results do not depend on it)."""
        _lib.check(self.lib.tg_tracker_set_slicing(self.tracker(), slice_steps))

    def slicing(self) -> int:
        v = ctypes.c_uint32()
        _lib.check(self.lib.tg_tracker_get_slicing(self.tracker(), ctypes.byref(v)))
        return v.value

    def tuning(self) -> dict:
        b, c, r = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        _lib.check(self.lib.tg_tracker_get_tuning(self.tracker(), ctypes.byref(b), ctypes.byref(c), ctypes.byref(r)))
        return {"blocks_per_sm": b.value, "compact_lanes": c.value, "compact_rounds": r.value}

    def device_scope(self):
        return _torch().cuda.device(self.device)

    def to_device(self, array: np.ndarray, dtype=None):
        """Upload a host array (through pinned memory) on this runtime's stream."""
        torch = _torch()
        host = torch.from_numpy(np.ascontiguousarray(array, dtype=dtype))
        with torch.cuda.stream(self.stream):
            return host.pin_memory().to(self.device, non_blocking=True)

    def empty(self, shape, dtype):
        torch = _torch()
        return torch.empty(shape, dtype=dtype, device=self.device)

    def pinned(self, shape, dtype) -> np.ndarray:
        """A page-locked host array (fast device-to-host copies)."""
        torch = _torch()
        t = torch.empty(shape, dtype=_TORCH_DTYPES[np.dtype(dtype)], pin_memory=True)
        return t.numpy().view(np.dtype(dtype))      # unsigned types live in same-size signed tensors

    def finish(self) -> None:
        """Wait for all work queued on this runtime's stream."""
        self.stream.synchronize()


def _destroy(fn, handle):
    try:
        fn(handle)
    except Exception:  # pragma: no cover - interpreter shutdown
        pass


_TORCH_DTYPES = {}


def _init_dtypes():
    try:
        import torch
    except ImportError:  # pragma: no cover
        return
    _TORCH_DTYPES.update({
        np.dtype(np.float32): torch.float32,
        np.dtype(np.uint32): torch.int32,
        np.dtype(np.int32): torch.int32,
        np.dtype(np.uint64): torch.int64,
        np.dtype(np.int64): torch.int64,
        np.dtype(np.uint8): torch.uint8,
    })


_init_dtypes()

_default_runtime = None


def default_runtime() -> CudaRuntime:
    """A process-wide runtime on the current device, created on first use."""
    global _default_runtime
    if _default_runtime is None:
        _default_runtime = CudaRuntime()
    return _default_runtime


class DeviceObject:
    """A library object (field or domain) owned by one runtime."""

    def __init__(self, handle: ctypes.c_void_p, destroy):
        self.handle = handle
        self._finalizer = weakref.finalize(self, _destroy, destroy, handle)

    def release(self):
        self._finalizer()
