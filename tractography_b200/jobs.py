"""Tracking jobs: prepared ``tg.tractogram`` requests and running many at once.

``prepare()`` performs the host-side half of the reference's
``tractography.tractogram`` (tractography/__init__.py:433-534): argument
validation, default local model / algorithm / domain, seed validation, and
one RNG seed per batch drawn from the algorithm in batch order.  ``run()``
tracks one prepared job; ``run_jobs()`` tracks any number of them in one
device-scheduled run (per code path one persistent launch, all on concurrent
streams), so small jobs share the GPU with large ones instead of each paying
for its own longest streamline.  Each job's result is identical to running
it alone.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field as dc_field
from pathlib import Path

import numpy as np

from . import _lib, local, nifti
from . import algorithm as algorithm_module
from . import domain as domain_module
from . import field as field_module
from . import seeds as seeds_module
from . import tracking
from .algorithm import BaseAlgorithm, to_struct
from .streamlines import ArraySequence, Tractogram


@dataclass
class Job:
    """A validated request: everything the device needs for one tg.tractogram call."""

    field: field_module.BaseField
    domain: domain_module.BaseDomain
    algorithm: BaseAlgorithm
    seeds: np.ndarray
    save_at: float
    n_steps: int
    min_points: int
    batch_size: int
    batch_rng_seeds: np.ndarray = dc_field(default_factory=lambda: np.zeros(0, np.uint32))
    philox_key: int = 0

    @property
    def n_seeds(self) -> int:
        return int(self.seeds.shape[0])


def _validate_algorithm(tracking_algorithm) -> None:
    if not isinstance(tracking_algorithm, BaseAlgorithm):
        raise TypeError("algorithm must be a BaseAlgorithm instance.")


def prepare(field, seeds, domain=None, algorithm=None, *, save_at: float = 1.0,
            maximum_streamline_length: float = 300.0, minimum_streamline_length: float = 0.0,
            batch_size: int = 50000, runtime=None):
    """Validate a tg.tractogram request; returns a :class:`Job` or an empty Tractogram."""
    if not np.isfinite(save_at) or save_at <= 0:
        raise ValueError("save_at must be finite and positive.")
    if not np.isfinite(maximum_streamline_length) or maximum_streamline_length < 0:
        raise ValueError("maximum_streamline_length must be finite and non-negative.")
    if not np.isfinite(minimum_streamline_length) or minimum_streamline_length < 0:
        raise ValueError("minimum_streamline_length must be finite and non-negative.")
    if minimum_streamline_length > maximum_streamline_length:
        raise ValueError("minimum_streamline_length must not exceed maximum_streamline_length.")
    if not isinstance(batch_size, (int, np.integer)) or batch_size <= 0:
        raise ValueError("batch_size must be a positive integer.")

    # The default domain (nonzero voxels of an image field) is built only when
    # no domain is given; the reference builds it eagerly (__init__.py:445-466),
    # which costs a pass over the whole field per call.
    if nifti.is_image(field):
        if field.ndim != 4:
            raise ValueError("The tracking image must be four-dimensional.")
        tracking_field = field_module.Image(field)
        image_affine = field.affine
        local_model = local.from_shape(field.shape)
    elif isinstance(field, field_module.BaseField):
        tracking_field = field
        local_model = local.from_shape((field.n_parameters,)) if algorithm is None else None
        image_affine = np.linalg.inv(field.inverse_affine) if isinstance(field, field_module.Image) else None
    else:
        raise TypeError("field must be a Nifti1Image or a BaseField instance.")

    if algorithm is None:
        tracking_algorithm = algorithm_module.Transport(local_model)
    else:
        _validate_algorithm(algorithm)
        tracking_algorithm = algorithm
    if tracking_algorithm.local_model.n_parameters != tracking_field.n_parameters:
        raise ValueError(
            "Algorithm local model parameter count does not match the field: "
            f"{tracking_algorithm.local_model.n_parameters} != {tracking_field.n_parameters}"
        )

    if isinstance(seeds, (int, np.integer)):
        if seeds < 0:
            raise ValueError("seeds must be a non-negative integer or an (n_seeds, 8) array.")
        n_seeds = int(seeds)
    elif isinstance(seeds, np.ndarray):
        seeds = seeds_module.validate_seed_array(seeds)
        n_seeds = len(seeds)
    else:
        raise TypeError("seeds must be a non-negative integer or an (n_seeds, 8) array.")

    if domain is not None and not (nifti.is_image(domain) or isinstance(domain, domain_module.BaseDomain)):
        raise TypeError("domain must be a BaseDomain, Nifti1Image, or None.")
    if n_seeds == 0:
        return Tractogram([], affine_to_rasmm=np.eye(4))

    if nifti.is_image(domain):
        tracking_domain = domain_module.Image(domain)
    elif domain is not None:
        tracking_domain = domain
    elif image_affine is not None:
        values = tracking_field.values
        tracking_domain = domain_module.Image(
            nifti.Nifti1Image(np.any(values != 0, axis=-1).astype(np.uint8), image_affine))
    else:
        raise ValueError(
            "A domain is required when the field is not an image field and "
            "does not provide an image-derived nonzero domain."
        )

    if isinstance(seeds, (int, np.integer)):
        seeds = domain_module.seed(tracking_domain, n_seeds, runtime=runtime)
    if len(seeds) == 0:
        return Tractogram([], affine_to_rasmm=np.eye(4))

    n_steps = tracking._n_steps(save_at, maximum_streamline_length)
    tracking._check_compatible(tracking_algorithm, tracking_field)
    n_batches = (len(seeds) + batch_size - 1) // batch_size
    batch_rng_seeds = np.array([tracking_algorithm.get_rng_seed() for _ in range(n_batches)], dtype=np.uint32)
    key = tracking_algorithm.philox_key() if tracking_algorithm.rng_mode() == _lib.RNG_PHILOX else 0
    return Job(field=tracking_field, domain=tracking_domain, algorithm=tracking_algorithm,
               seeds=np.ascontiguousarray(seeds, dtype=np.float32), save_at=float(save_at), n_steps=n_steps,
               min_points=int(np.ceil(minimum_streamline_length / save_at)), batch_size=int(batch_size),
               batch_rng_seeds=batch_rng_seeds, philox_key=key)


def _to_tractogram(job: Job, result: tracking.TrackResult) -> Tractogram:
    keep = result.lengths > job.min_points
    return Tractogram(result.streamlines(keep), affine_to_rasmm=np.eye(4))


def run(job: Job, runtime) -> Tractogram:
    """Track one prepared job with the single-job persistent tracker."""
    result = tracking.track_packed(job.algorithm, job.domain, job.field, job.seeds, save_at=job.save_at,
                                   n_steps=job.n_steps, batch_size=job.batch_size,
                                   batch_rng_seeds=job.batch_rng_seeds, runtime=runtime,
                                   philox_key=job.philox_key)
    return _to_tractogram(job, result)


def write(job: Job, filename, runtime, seeds_per_pass: int = 1_000_000, affine=None) -> int:
    """Track a prepared job and stream its streamlines to a ``.tck`` or
    ``.trx`` file; returns the number of streamlines written.

    The reference's command line does this for TRX by calling
    ``tracking.tractogram`` per batch and appending the kept streamlines to a
    memory-mapped writer (tractography/cli/tractogram.py:81-139).  Here the
    seeds go to the tracker ``seeds_per_pass`` at a time (rounded to whole
    batches, so every batch keeps its RNG seed and per-batch stream ids) and
    each pass's packed output is appended to the streaming writer with the
    minimum-length filter applied as a mask: host memory stays bounded by
    one pass and no per-streamline Python objects are made.  The file holds
    exactly the streamlines ``run`` returns, in the same order.
    """
    from .streamlines import TckWriter, TrxWriter

    suffix = Path(filename).suffix.lower()
    if suffix == ".tck":
        writer = TckWriter(filename, affine)
    elif suffix == ".trx":
        writer = TrxWriter(filename, affine)
    else:
        raise ValueError(f"Unknown tractogram file type: {suffix or filename}")
    per_pass = max(1, int(seeds_per_pass) // job.batch_size) * job.batch_size
    written = 0
    with writer:
        for lo in range(0, job.n_seeds, per_pass):
            hi = min(job.n_seeds, lo + per_pass)
            b0, b1 = lo // job.batch_size, (hi + job.batch_size - 1) // job.batch_size
            result = tracking.track_packed(job.algorithm, job.domain, job.field, job.seeds[lo:hi],
                                           save_at=job.save_at, n_steps=job.n_steps, batch_size=job.batch_size,
                                           batch_rng_seeds=job.batch_rng_seeds[b0:b1], runtime=runtime,
                                           philox_key=job.philox_key, seed_offset=lo)
            keep = result.lengths > job.min_points
            writer.append(result.points, result.lengths[keep], result.offsets[keep])
            written += int(keep.sum())
    return written


class JobsResult:
    """Packed output of a multi-job run: per-job slices of one point buffer."""

    def __init__(self, points, offsets, lengths, steps, bounds):
        self.points = points
        self.offsets = offsets
        self.lengths = lengths
        self.steps = int(steps)
        self.bounds = bounds

    def job(self, j: int) -> tracking.TrackResult:
        a, b = self.bounds[j], self.bounds[j + 1]
        return tracking.TrackResult(self.points, self.offsets[a:b], self.lengths[a:b], 0)


def run_jobs_packed(jobs, runtime) -> JobsResult:
    """Track all jobs in one device-scheduled run; returns the packed result."""
    jobs = list(jobs)
    structs = (_lib.Job * max(1, len(jobs)))()
    keep_alive = []
    bounds = [0]
    with runtime.device_scope():
        for j, job in enumerate(jobs):
            d_handle, f_handle = tracking._handles(job.algorithm, job.domain, job.field, runtime)
            seeds = np.ascontiguousarray(job.seeds, dtype=np.float32)
            rng = np.ascontiguousarray(job.batch_rng_seeds, dtype=np.uint32)
            keep_alive += [seeds, rng]
            s = structs[j]
            s.domain, s.field = d_handle, f_handle
            s.algorithm = to_struct(job.algorithm, 0, job.philox_key, 0)
            s.seeds = seeds.ctypes.data
            s.n_seeds = job.n_seeds
            s.batch_size = job.batch_size
            s.batch_rng_seeds = rng.ctypes.data
            s.save_at = job.save_at
            s.n_steps = job.n_steps
            bounds.append(bounds[-1] + job.n_seeds)
        n = bounds[-1]
        lengths = np.empty(max(1, n), dtype=np.uint32)
        offsets = np.empty(max(1, n), dtype=np.uint64)
        total = ctypes.c_uint64()
        steps = ctypes.c_uint64()
        _lib.check(runtime.lib.tg_tracker_run_jobs(
            runtime.tracker(), structs, len(jobs), 1, lengths.ctypes.data_as(ctypes.c_void_p),
            offsets.ctypes.data_as(ctypes.c_void_p), ctypes.byref(total), ctypes.byref(steps),
            ctypes.c_void_p(runtime.stream_handle)))
        points = runtime.pinned((int(total.value), 3), np.float32) if total.value else np.empty((0, 3), np.float32)
        if total.value:
            _lib.check(runtime.lib.tg_tracker_copy_points(
                runtime.tracker(), points.ctypes.data_as(ctypes.c_void_p), 0, total.value, 1,
                ctypes.c_void_p(runtime.stream_handle)))
    return JobsResult(points, offsets[:n].astype(np.int64), lengths[:n].astype(np.int64), steps.value,
                      np.asarray(bounds))


def run_jobs(jobs, runtime=None) -> list:
    """Track prepared jobs together; returns one Tractogram per job, in order."""
    from .runtime import default_runtime

    runtime = runtime or default_runtime()
    jobs = list(jobs)
    if not jobs:
        return []
    result = run_jobs_packed(jobs, runtime)
    return [_to_tractogram(job, result.job(j)) for j, job in enumerate(jobs)]


def empty_streamlines() -> ArraySequence:
    return ArraySequence()
