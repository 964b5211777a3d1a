"""Continuous-batching tracking server (no reference counterpart).

The reference tracks one ``tg.tractogram`` call at a time.  ``Server``
keeps fields, domains and surfaces resident on the GPU and runs many
requests at once through the library's epoch scheduler (tg_server_*): every
epoch, one persistent launch per code path resumes the streamlines carried
over from the previous epoch and takes new seeds from the request queues;
requests that arrive while others run join between epochs, as memory and
request slots free up.  A request is one ``tg.tractogram`` job; its result is
identical to the same job tracked alone.

    server = Server(hbm_budget_bytes=150e9)
    rid = server.submit(jobs.prepare(fod, seeds, algorithm=alg))
    while not done:
        for rid in server.poll():
            tractogram = server.result(rid)
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib, jobs, tracking
from .algorithm import to_struct
from .streamlines import ArraySequence, Tractogram


@dataclass
class ServerStats:
    steps: int
    epochs: int
    busy_seconds: float          # host wall time of the epochs
    reserved_bytes: int
    kernel_seconds: float = 0.0  # device time of the epochs' tracking launches
    between_seconds: float = 0.0 # from their end to the harvest (read-back, host bookkeeping)
    harvest_seconds: float = 0.0 # device time of moving finished streamlines to their results


class Server:
    """Admission by HBM budget, epoch scheduling, results by request id.

    Args:
        runtime: ``CudaRuntime`` whose device runs the server (default: the
            process-wide runtime).
        hbm_budget_bytes: device memory the server may hold for its point
            pool, request buffers and unclaimed results.
        pool_points: capacity of the shared point pool (0: 32M points).
        epoch_steps: loop iterations per lane per epoch.
        max_requests: admitted requests at a time.
        epoch_seconds: device-clock budget of an epoch (0: epoch_steps
            alone ends it); every code path stops at the same deadline.
        reserve_bytes: device memory mapped into the server's pool at
            creation for request buffers and results (default: the budget
            less the point pool, at most 90 % of the free memory); 0 maps
            on demand, which costs time between epochs.
    """

    def __init__(self, runtime=None, *, hbm_budget_bytes: float = 150e9, pool_points: int = 0,
                 epoch_steps: int = 1024, max_requests: int = 256, epoch_seconds: float = 0.0,
                 reserve_bytes: int | None = None):
        from .runtime import default_runtime

        self.runtime = runtime or default_runtime()
        self.lib = self.runtime.lib
        self._handle = ctypes.c_void_p()
        with self.runtime.device_scope():
            _lib.check(self.lib.tg_server_create(int(hbm_budget_bytes), int(pool_points), int(epoch_steps),
                                                 int(max_requests), ctypes.byref(self._handle)))
            if epoch_seconds:
                _lib.check(self.lib.tg_server_set_epoch_time(self._handle, float(epoch_seconds)))
            if reserve_bytes is None:
                import torch

                free, _ = torch.cuda.mem_get_info(self.runtime.device)
                pool = (pool_points or (32 << 20)) * 12
                reserve_bytes = int(max(0.0, min(hbm_budget_bytes - pool, 0.9 * free - pool)))
            if reserve_bytes > 0 and self.lib.tg_server_reserve(self._handle, int(reserve_bytes)) != 0:
                # the reservation only saves time: without it the pool maps
                # memory as requests need it
                import warnings

                message = self.lib.tg_last_error().decode(errors="replace")
                warnings.warn(f"server memory reservation of {reserve_bytes} bytes failed: {message}")
        self._jobs = {}
        self._arrays = {}
        self._ids = (ctypes.c_uint64 * 1024)()

    def close(self) -> None:
        if self._handle:
            with self.runtime.device_scope():
                self.lib.tg_server_destroy(self._handle)
            self._handle = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):  # pragma: no cover - best effort
        try:
            self.close()
        except Exception:
            pass

    def submit(self, job: jobs.Job) -> int:
        """Queue one prepared job (``jobs.prepare``); returns its request id."""
        s = _lib.Job()
        with self.runtime.device_scope():
            d_handle, f_handle = tracking._handles(job.algorithm, job.domain, job.field, self.runtime)
            seeds = np.ascontiguousarray(job.seeds, dtype=np.float32)
            rng = np.ascontiguousarray(job.batch_rng_seeds, dtype=np.uint32)
            s.domain, s.field = d_handle, f_handle
            s.algorithm = to_struct(job.algorithm, 0, job.philox_key, 0)
            s.seeds = seeds.ctypes.data
            s.n_seeds = job.n_seeds
            s.batch_size = job.batch_size
            s.batch_rng_seeds = rng.ctypes.data
            s.save_at = job.save_at
            s.n_steps = job.n_steps
            rid = ctypes.c_uint64()
            _lib.check(self.lib.tg_server_submit(self._handle, ctypes.byref(s), ctypes.byref(rid)))
        # the server reads the host seeds at admission: keep them alive until the result is taken
        self._jobs[rid.value] = job
        self._arrays[rid.value] = (seeds, rng)
        return rid.value

    def poll(self) -> list[int]:
        """Run one epoch; returns the ids of requests that finished."""
        n, active, pending = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint32()
        with self.runtime.device_scope():
            _lib.check(self.lib.tg_server_poll(self._handle, self._ids, len(self._ids), ctypes.byref(n),
                                               ctypes.byref(active), ctypes.byref(pending)))
        self.active, self.pending = active.value, pending.value
        return [int(self._ids[i]) for i in range(n.value)]

    def result_size(self, request_id: int):
        n, p, t = ctypes.c_uint32(), ctypes.c_uint64(), ctypes.c_double()
        _lib.check(self.lib.tg_server_result_size(self._handle, request_id, ctypes.byref(n), ctypes.byref(p),
                                                  ctypes.byref(t)))
        return n.value, p.value, t.value

    def take(self, request_id: int, points: bool = True):
        """Result of a finished request: (points (P, 3) or None, per-seed
        offsets into points, per-seed lengths, seconds from submission to
        completion); releases it on the device."""
        n, p, seconds = self.result_size(request_id)
        lengths = np.empty(max(1, n), np.uint32)
        offsets = np.empty(max(1, n), np.uint64)
        pts = np.empty((max(1, p), 3), np.float32) if points else None
        with self.runtime.device_scope():
            _lib.check(self.lib.tg_server_take(self._handle, request_id, lengths.ctypes.data_as(ctypes.c_void_p),
                                               offsets.ctypes.data_as(ctypes.c_void_p),
                                               pts.ctypes.data_as(ctypes.c_void_p) if points else None))
        self._jobs.pop(request_id, None)
        self._arrays.pop(request_id, None)
        return (pts[:p] if points else None), offsets[:n].astype(np.int64), lengths[:n].astype(np.int64), seconds

    def result(self, request_id: int) -> Tractogram:
        """The finished request as a Tractogram (the minimum-length filter of
        tg.tractogram applied), released on the device."""
        job = self._jobs.get(request_id)
        points, offsets, lengths, _ = self.take(request_id)
        keep = lengths > (job.min_points if job is not None else 0)
        return Tractogram(ArraySequence(points, offsets[keep], lengths[keep]), affine_to_rasmm=np.eye(4))

    def stats(self) -> ServerStats:
        steps, epochs, busy, reserved = ctypes.c_uint64(), ctypes.c_uint64(), ctypes.c_double(), ctypes.c_uint64()
        _lib.check(self.lib.tg_server_stats(self._handle, ctypes.byref(steps), ctypes.byref(epochs),
                                            ctypes.byref(busy), ctypes.byref(reserved)))
        kernel, between, harvest = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _lib.check(self.lib.tg_server_timing(self._handle, ctypes.byref(kernel), ctypes.byref(between),
                                             ctypes.byref(harvest)))
        return ServerStats(steps.value, epochs.value, busy.value, reserved.value, kernel.value, between.value,
                           harvest.value)

    def drain(self) -> dict:
        """Poll until every submitted request finished; returns {id: Tractogram}."""
        out = {}
        idle = 0
        polls = 0
        while self._jobs:
            polls += 1
            if polls > 10_000_000:
                raise RuntimeError("requests stopped making progress")
            finished = self.poll()
            for rid in finished:
                out[rid] = self.result(rid)
            idle = 0 if finished or self.active else idle + 1
            if idle > 2:
                raise RuntimeError("requests remain that the server cannot admit")
        return out
