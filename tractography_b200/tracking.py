"""Low-level streamline tracking (reference ``tractography/tracking.py:22-178``).

``tractogram()`` keeps the reference's signature and semantics: every seed
is advanced by the algorithm while it stays inside the domain and the field
can be evaluated; a point is recorded every ``save_at`` of path length
(back-interpolated to the exact save position), the seed itself first, up
to ``floor(maximum_streamline_length / save_at)`` points.

Execution differs from the reference: no source assembly or per-call
compilation, the field and domain stay resident on the device, and seeds are
tracked by the persistent kernel whose packed output is copied back once.
``tractogram_dense()`` runs the one-thread-per-seed kernel with the
reference's dense output layout.
"""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .algorithm import BaseAlgorithm, to_struct
from .domain import BaseDomain
from .domain import Image as ImageDomain
from .domain import Mesh as MeshDomain
from .field import BaseField
from .field import Image as ImageField
from .local import model_id
from .seeds import validate_seed_array
from .streamlines import ArraySequence, Tractogram


class TrackResult:
    """Packed output of one tracker run."""

    def __init__(self, points, offsets, lengths, steps):
        self.points = points
        self.offsets = offsets
        self.lengths = lengths
        self.steps = int(steps)

    def streamlines(self, keep=None) -> ArraySequence:
        if keep is None:
            return ArraySequence(self.points, self.offsets, self.lengths)
        return ArraySequence(self.points, self.offsets[keep], self.lengths[keep])


def _check_compatible(algorithm: BaseAlgorithm, field: BaseField) -> None:
    if algorithm.local_model.n_parameters != field.n_parameters:
        raise ValueError(
            "Incompatible local model and field, they do not have the "
            "same number of parameters: "
            f"{algorithm.local_model.n_parameters} != {field.n_parameters}"
        )


def _n_steps(save_at: float, maximum_streamline_length: float) -> int:
    n_steps = int(np.floor(maximum_streamline_length / save_at))
    if n_steps <= 0:
        # The reference allocates an empty point buffer here and fails
        # (opencl.py:323-324).
        raise ValueError("nbytes must be positive.")
    return n_steps


def _handles(algorithm, domain, field, runtime):
    if not isinstance(domain, (ImageDomain, MeshDomain)):
        raise NotImplementedError(f"{type(domain).__name__} has no compiled CUDA code path")
    if not isinstance(field, ImageField):
        raise NotImplementedError(f"{type(field).__name__} has no compiled CUDA code path")
    mid = model_id(algorithm.local_model)
    return domain.device(runtime), field.device(runtime, mid)


def track_packed(algorithm: BaseAlgorithm, domain: BaseDomain, field: BaseField, seeds: np.ndarray, *,
                 save_at: float, n_steps: int, batch_size: int, batch_rng_seeds, runtime,
                 philox_key: int = 0, seed_offset: int = 0) -> TrackResult:
    """Track all seeds with one persistent-tracker run.

    Seed ``i`` is tracked with the stream of batch ``i // batch_size``
    (seed ``batch_rng_seeds[b]``) and stream id ``i % batch_size``.
    """
    n = int(seeds.shape[0])
    batch_rng_seeds = np.ascontiguousarray(batch_rng_seeds, dtype=np.uint32)
    if len(batch_rng_seeds) != (n + batch_size - 1) // batch_size:
        raise ValueError("one rng seed per batch is required")
    lengths = np.empty(n, dtype=np.uint32)
    offsets = np.empty(n, dtype=np.uint64)
    total = ctypes.c_uint64()
    steps = ctypes.c_uint64()
    with runtime.device_scope():
        d_handle, f_handle = _handles(algorithm, domain, field, runtime)
        a = to_struct(algorithm, 0, philox_key, seed_offset)
        seeds = np.ascontiguousarray(seeds, dtype=np.float32)
        _lib.check(runtime.lib.tg_tracker_run(
            runtime.tracker(), ctypes.byref(a), d_handle, f_handle, seeds.ctypes.data_as(ctypes.c_void_p), 1, n,
            int(batch_size), batch_rng_seeds.ctypes.data_as(ctypes.c_void_p), float(save_at), int(n_steps),
            lengths.ctypes.data_as(ctypes.c_void_p), offsets.ctypes.data_as(ctypes.c_void_p),
            ctypes.byref(total), ctypes.byref(steps), ctypes.c_void_p(runtime.stream_handle)))
        points = runtime.pinned((int(total.value), 3), np.float32) if total.value else np.empty((0, 3), np.float32)
        if total.value:
            _lib.check(runtime.lib.tg_tracker_copy_points(
                runtime.tracker(), points.ctypes.data_as(ctypes.c_void_p), 0, total.value, 1,
                ctypes.c_void_p(runtime.stream_handle)))
    return TrackResult(points, offsets.astype(np.int64), lengths.astype(np.int64), steps.value)


def tractogram(algorithm: BaseAlgorithm, domain: BaseDomain, field: BaseField, seeds: np.ndarray,
               save_at: float = 1.0, maximum_streamline_length: float = 300.0, runtime=None) -> Tractogram:
    """Track streamlines from (n, 8) position-and-orientation seeds.

    Raises:
        ValueError: if the local model and field have different parameter
            counts (tracking.py:72-78).
    """
    seeds = validate_seed_array(seeds)
    _check_compatible(algorithm, field)
    n_seeds = seeds.shape[0]
    if n_seeds == 0:
        return Tractogram([], affine_to_rasmm=np.eye(4))
    from .runtime import default_runtime

    runtime = runtime or default_runtime()
    n_steps = _n_steps(save_at, maximum_streamline_length)
    rng_seed = algorithm.get_rng_seed()
    key = algorithm.philox_key() if algorithm.rng_mode() == _lib.RNG_PHILOX else 0
    result = track_packed(algorithm, domain, field, seeds, save_at=save_at, n_steps=n_steps, batch_size=n_seeds,
                          batch_rng_seeds=[rng_seed], runtime=runtime, philox_key=key)
    return Tractogram(result.streamlines(), affine_to_rasmm=np.eye(4))


def tractogram_dense(algorithm: BaseAlgorithm, domain: BaseDomain, field: BaseField, seeds: np.ndarray,
                     save_at: float = 1.0, maximum_streamline_length: float = 300.0, runtime=None,
                     rng_seed: int | None = None, philox_key: int | None = None):
    """The reference kernel contract: dense (n, n_steps, 4) points and lengths.

    Runs one thread per seed (the plain one-launch form) and returns the
    host arrays the reference's kernel writes (tracking.py:152-176).
    """
    seeds = validate_seed_array(seeds)
    _check_compatible(algorithm, field)
    n = seeds.shape[0]
    from .runtime import default_runtime

    runtime = runtime or default_runtime()
    n_steps = _n_steps(save_at, maximum_streamline_length)
    if rng_seed is None:
        rng_seed = algorithm.get_rng_seed()
    if philox_key is None:
        philox_key = algorithm.philox_key() if algorithm.rng_mode() == _lib.RNG_PHILOX else 0
    out = np.zeros((n, n_steps, 4), dtype=np.float32)
    lengths = np.zeros(n, dtype=np.uint32)
    if n == 0:
        return out, lengths
    with runtime.device_scope():
        d_handle, f_handle = _handles(algorithm, domain, field, runtime)
        a = to_struct(algorithm, rng_seed, philox_key, 0)
        _lib.check(runtime.lib.tg_tractogram_host(
            ctypes.byref(a), d_handle, f_handle, seeds.ctypes.data_as(ctypes.c_void_p), n, float(save_at), n_steps,
            out.ctypes.data_as(ctypes.c_void_p), lengths.ctypes.data_as(ctypes.c_void_p),
            ctypes.c_void_p(runtime.stream_handle)))
    return out, lengths


def tod(algorithm: BaseAlgorithm, domain: BaseDomain, field: BaseField, image, n_seeds: int,
        maximum_streamline_length: float = 300.0, runtime=None, *, stats: dict | None = None):
    """Track orientation distribution as lmax-8 SH coefficients (tracking.py:181-385).

    ``n_seeds`` seeds are drawn on the domain boundary (``domain.seed``'s
    sampler, stream rng_init(rng_seed, i) with rng_seed = the algorithm's next
    seed); each track is integrated for at most
    floor(maximum_streamline_length / step_size) iterations and the real SH
    basis of its orientation at every iteration is added to the output voxel
    nearest the point on ``image``'s grid.  Each nonempty voxel is normalised
    to unit integral.  Returns an image of shape image.shape + (45,).  When
    ``stats`` is a dict, stats["steps"] receives the number of tracking
    iterations that passed the domain and field tests.
    """
    from .nifti import Nifti1Image
    from .utils import normalize_odf

    _check_compatible(algorithm, field)
    if not isinstance(n_seeds, (int, np.integer)) or n_seeds < 0:
        raise ValueError("n_seeds must be a non-negative integer.")
    if not np.isfinite(maximum_streamline_length) or maximum_streamline_length < 0:
        raise ValueError("maximum_streamline_length must be finite and non-negative.")
    if len(image.shape) != 3:
        raise ValueError("The output image description must be 3D.")
    output_shape = tuple(int(size) for size in image.shape)
    affine = np.asarray(image.affine if image.affine is not None else np.eye(4), dtype=np.float64)
    inverse_affine = np.ascontiguousarray(np.linalg.inv(affine), dtype=np.float32)
    step_size = float(algorithm.step_size)
    if not np.isfinite(step_size) or step_size <= 0:
        raise ValueError("algorithm.step_size must be finite and positive.")
    n_steps = int(np.floor(maximum_streamline_length / step_size))
    header = getattr(image, "header", None)
    if n_seeds > 0 and n_steps > 0:
        from .runtime import default_runtime

        runtime = runtime or default_runtime()
        import torch

        v4, f4, cumulative = domain.boundary_arrays()
        with runtime.device_scope():
            d_handle, f_handle = _handles(algorithm, domain, field, runtime)
            a = to_struct(algorithm, algorithm.get_rng_seed(),
                          algorithm.philox_key() if algorithm.rng_mode() == _lib.RNG_PHILOX else 0, 0)
            dv, df, dc = runtime.to_device(v4), runtime.to_device(f4), runtime.to_device(cumulative)
            with torch.cuda.stream(runtime.stream):    # zeroed on the stream the kernel runs on
                coefficients = torch.zeros(output_shape + (45,), dtype=torch.float32, device=runtime.device)
                steps = torch.zeros((1,), dtype=torch.int64, device=runtime.device)
            dims = np.asarray(output_shape, dtype=np.uint32)
            _lib.check(runtime.lib.tg_tod(
                ctypes.byref(a), d_handle, f_handle, ctypes.c_void_p(dv.data_ptr()), len(v4),
                ctypes.c_void_p(df.data_ptr()), ctypes.c_void_p(dc.data_ptr()), len(f4), int(n_seeds), n_steps,
                dims.ctypes.data_as(ctypes.c_void_p), inverse_affine.ctypes.data_as(ctypes.c_void_p),
                ctypes.c_void_p(coefficients.data_ptr()), ctypes.c_void_p(steps.data_ptr()),
                ctypes.c_void_p(runtime.stream_handle)))
            # normalize_odf on the device, in its float64 operations
            # (c / sqrt(4 pi) / c0, rounded to float32; zero where c0 == 0),
            # then one copy of the result to page-locked host memory
            out = runtime.pinned(output_shape + (45,), np.float32)
            with torch.cuda.stream(runtime.stream):
                c0 = coefficients[..., :1]
                normalized = torch.where(c0 != 0, (coefficients.double() / np.sqrt(4 * np.pi) / c0.double()).float(),
                                         torch.zeros((), dtype=torch.float32, device=coefficients.device))
                torch.from_numpy(out).copy_(normalized)
                if stats is not None:
                    stats["steps"] = int(steps.item())
            return Nifti1Image(out, affine, header)
    raw = np.zeros(output_shape + (45,), dtype=np.float32)
    return Nifti1Image(normalize_odf(raw).astype(np.float32), affine, header)


def connectome(algorithm: BaseAlgorithm, domain: BaseDomain, field: BaseField, n_seeds: int,
               maximum_streamline_length: float = 300.0, minimum_streamline_length: float = 0.0, runtime=None, *,
               stats: dict | None = None):
    """Directed piecewise-linear boundary connectome (tracking.py:388-602).

    Tracks start on the domain boundary (``domain.seed``'s sampler); when a
    track stops for any reason its final segment is tested against the
    boundary BVH, and a track that moved at least ``minimum_streamline_length``
    and hit the boundary adds the outer product of its start and end
    barycentric weights at the two triangles' vertices.  Returns a float32
    (n_vertices, n_vertices) CSR matrix over ``domain.boundary.vertices``.
    ``stats`` as for :func:`tod`.
    """
    from scipy.sparse import coo_matrix, csr_matrix

    _check_compatible(algorithm, field)
    if not isinstance(n_seeds, (int, np.integer)) or n_seeds < 0:
        raise ValueError("n_seeds must be a non-negative integer.")
    if not np.isfinite(maximum_streamline_length) or maximum_streamline_length < 0:
        raise ValueError("maximum_streamline_length must be finite and non-negative.")
    if not np.isfinite(minimum_streamline_length) or minimum_streamline_length < 0:
        raise ValueError("minimum_streamline_length must be finite and non-negative.")
    if minimum_streamline_length > maximum_streamline_length:
        raise ValueError("minimum_streamline_length must not exceed maximum_streamline_length.")
    n_vertices = len(domain.boundary.vertices)
    if n_seeds == 0 or n_vertices == 0:
        return csr_matrix((n_vertices, n_vertices), dtype=np.float32)
    step_size = float(algorithm.step_size)
    if not np.isfinite(step_size) or step_size <= 0:
        raise ValueError("algorithm.step_size must be finite and positive.")
    n_steps = int(np.floor(maximum_streamline_length / step_size))
    if n_steps == 0:
        return csr_matrix((n_vertices, n_vertices), dtype=np.float32)
    from .runtime import default_runtime

    runtime = runtime or default_runtime()
    import torch

    v4, f4, cumulative = domain.boundary_arrays()
    with runtime.device_scope():
        d_handle, f_handle = _handles(algorithm, domain, field, runtime)
        b_handle = domain.boundary_bvh().device(runtime)
        a = to_struct(algorithm, algorithm.get_rng_seed(),
                      algorithm.philox_key() if algorithm.rng_mode() == _lib.RNG_PHILOX else 0, 0)
        dv, df, dc = runtime.to_device(v4), runtime.to_device(f4), runtime.to_device(cumulative)
        rows = runtime.empty((9 * int(n_seeds),), torch.int32)
        cols = runtime.empty((9 * int(n_seeds),), torch.int32)
        weights = runtime.empty((9 * int(n_seeds),), torch.float32)
        with torch.cuda.stream(runtime.stream):        # zeroed on the stream the kernel runs on
            steps = torch.zeros((1,), dtype=torch.int64, device=runtime.device)
        _lib.check(runtime.lib.tg_connectome(
            ctypes.byref(a), d_handle, f_handle, b_handle, ctypes.c_void_p(dv.data_ptr()), len(v4),
            ctypes.c_void_p(df.data_ptr()), ctypes.c_void_p(dc.data_ptr()), len(f4), int(n_seeds), n_steps,
            float(minimum_streamline_length), ctypes.c_void_p(rows.data_ptr()), ctypes.c_void_p(cols.data_ptr()),
            ctypes.c_void_p(weights.data_ptr()), ctypes.c_void_p(steps.data_ptr()),
            ctypes.c_void_p(runtime.stream_handle)))
        with torch.cuda.stream(runtime.stream):
            rows, cols, weights = rows.cpu().numpy(), cols.cpu().numpy(), weights.cpu().numpy()
            if stats is not None:
                stats["steps"] = int(steps.item())
    return contributions_to_matrix(rows, cols, weights, n_vertices)


def contributions_to_matrix(rows, cols, weights, n_vertices):
    """Sum the kernel's (row, column, weight) contributions into a CSR matrix."""
    from scipy.sparse import coo_matrix, csr_matrix

    valid = rows >= 0
    if not np.any(valid):
        return csr_matrix((n_vertices, n_vertices), dtype=np.float32)
    matrix = coo_matrix((weights[valid], (rows[valid], cols[valid])), shape=(n_vertices, n_vertices),
                        dtype=np.float32).tocsr()
    matrix.sum_duplicates()
    return matrix
