"""tractography_b200 -- streamline tracking of cronos-inria/tractography on B200.

A drop-in for the reference's tracking path: the public ``tractogram``
function, the ``algorithm`` (Transport, Diffusion), ``local``
(RealSymmetricSphericalHarmonics, DiffusionTensorImaging), ``field``,
``domain`` and ``seeds`` modules and ``.tck`` output keep the reference's
names, arguments and errors; the OpenCL backend is replaced by compiled
sm_100a CUDA kernels behind the C ABI of ``include/tractography_b200.h``.
``jobs.run_jobs`` tracks many requests in one device-scheduled run.
"""

from __future__ import annotations

from . import algorithm as algorithm_module
from . import core, jobs, local, nifti, streamlines, tracking, utils
from . import domain as domain_module
from . import field as field_module
from . import seeds
from .nifti import Nifti1Image
from .opencl import BufferAccess, OpenCLRuntime
from .runtime import CudaRuntime
from .streamlines import ArraySequence, TckWriter, Tractogram, TrxWriter, load_tck, load_trx, save_tck, save_trx

algorithm = algorithm_module
domain = domain_module
field = field_module
seeds_module = seeds

__all__ = [
    "ArraySequence", "BufferAccess", "CudaRuntime", "Nifti1Image", "OpenCLRuntime", "TckWriter", "Tractogram", "TrxWriter",
    "load_trx", "save_trx",
    "algorithm", "core", "domain", "field", "jobs", "load_tck", "local", "nifti", "save_tck", "seeds",
    "connectome", "streamlines", "tod", "tracking", "tractogram", "utils", "write_tractogram",
]


def connectome(field, n_seeds: int = 1000000, domain=None, algorithm=None, segmentation=None, *,
               distance_upper_bound: float = 4.0, maximum_streamline_length: float = 300.0,
               minimum_streamline_length: float = 0.0, runtime=None):
    """Boundary or region connectome (__init__.py:45-214).

    Without ``segmentation``: the directed boundary-vertex connectome (CSR)
    and the vertex indices.  With a segmentation of positive labels: boundary
    vertices are assigned to their nearest labelled voxel within
    ``distance_upper_bound`` and the matrix is aggregated by region (dense,
    not symmetrised), with the labels."""
    import numpy as np
    from scipy.sparse import csr_matrix
    from scipy.spatial import cKDTree

    from .nifti import apply_affine

    if not isinstance(n_seeds, (int, np.integer)) or n_seeds < 0:
        raise ValueError("n_seeds must be a non-negative integer.")
    if not np.isfinite(distance_upper_bound) or distance_upper_bound < 0:
        raise ValueError("distance_upper_bound must be finite and non-negative.")
    if not np.isfinite(maximum_streamline_length) or maximum_streamline_length < 0:
        raise ValueError("maximum_streamline_length must be finite and non-negative.")
    if not np.isfinite(minimum_streamline_length) or minimum_streamline_length < 0:
        raise ValueError("minimum_streamline_length must be finite and non-negative.")
    if minimum_streamline_length > maximum_streamline_length:
        raise ValueError("minimum_streamline_length must not exceed maximum_streamline_length.")
    seg_data = labels = None
    if segmentation is not None:
        if not nifti.is_image(segmentation):
            raise TypeError("segmentation must be a Nifti1Image or None.")
        seg_data = np.asanyarray(segmentation.dataobj)
        if seg_data.ndim != 3:
            raise ValueError("Segmentation image must be three-dimensional.")
        labels = np.unique(seg_data[seg_data > 0])
        labels = labels[labels > 0]
        if len(labels) == 0:
            return np.zeros((0, 0), dtype=np.float32), labels
    domain_image = None
    local_model = None
    if nifti.is_image(field):
        if field.ndim != 4:
            raise ValueError("The tracking image must be four-dimensional.")
        tracking_field = field_module.Image(field)
        domain_image = Nifti1Image(np.any(np.asanyarray(field.dataobj) != 0, axis=-1).astype(np.uint8), field.affine)
        local_model = local.from_shape(field.shape)
    elif isinstance(field, field_module.BaseField):
        tracking_field = field
        local_model = local.from_shape((field.n_parameters,)) if algorithm is None else None
        if isinstance(field, field_module.Image):
            domain_image = Nifti1Image(np.any(field.values != 0, axis=-1).astype(np.uint8),
                                       np.linalg.inv(field.inverse_affine))
    else:
        raise TypeError("field must be a Nifti1Image or a BaseField instance.")
    if algorithm is None:
        tracking_algorithm = algorithm_module.Transport(local_model)
    else:
        jobs._validate_algorithm(algorithm)
        tracking_algorithm = algorithm
    if tracking_algorithm.local_model.n_parameters != tracking_field.n_parameters:
        raise ValueError(
            "Algorithm local model parameter count does not match the field: "
            f"{tracking_algorithm.local_model.n_parameters} != {tracking_field.n_parameters}"
        )
    if domain is not None and not (nifti.is_image(domain) or isinstance(domain, domain_module.BaseDomain)):
        raise TypeError("domain must be a BaseDomain, Nifti1Image, or None.")
    if nifti.is_image(domain):
        tracking_domain = domain_module.Image(domain)
    elif domain is not None:
        tracking_domain = domain
    elif domain_image is not None:
        if not np.any(np.asanyarray(domain_image.dataobj) != 0):
            if labels is None:
                return csr_matrix((0, 0), dtype=np.float32), np.empty(0, dtype=np.intp)
            return np.zeros((len(labels), len(labels)), dtype=np.float32), labels
        tracking_domain = domain_module.Image(domain_image)
    else:
        raise ValueError("A domain is required when the field is not an image field.")
    boundary_matrix = tracking.connectome(tracking_algorithm, tracking_domain, tracking_field, n_seeds,
                                          maximum_streamline_length=maximum_streamline_length,
                                          minimum_streamline_length=minimum_streamline_length, runtime=runtime)
    if labels is None:
        return boundary_matrix, np.arange(boundary_matrix.shape[0], dtype=np.intp)
    voxel_indices = np.argwhere(seg_data > 0)
    affine = segmentation.affine if segmentation.affine is not None else np.eye(4)
    vertices = tracking_domain.boundary.vertices
    distances, nearest = cKDTree(apply_affine(affine, voxel_indices)).query(
        vertices, distance_upper_bound=distance_upper_bound)
    distances = np.asarray(distances).reshape(-1)
    nearest = np.asarray(nearest, dtype=np.intp).reshape(-1)
    assigned = np.isfinite(distances)
    label_index = {label: k for k, label in enumerate(labels)}
    vertex_labels = np.zeros(len(vertices), dtype=np.intp)
    hit = voxel_indices[nearest[assigned]]
    vertex_labels[assigned] = np.fromiter((label_index[x] for x in seg_data[hit[:, 0], hit[:, 1], hit[:, 2]]),
                                          dtype=np.intp, count=int(np.count_nonzero(assigned)))
    selected = np.flatnonzero(assigned)
    assignment = csr_matrix((np.ones(len(selected), dtype=np.float32), (vertex_labels[selected], selected)),
                            shape=(len(labels), len(vertex_labels)))
    matrix = (assignment @ boundary_matrix @ assignment.T).tocsr()
    return matrix.toarray(), labels


def tod(field, n_seeds: int = 1000000, domain=None, algorithm=None, *, maximum_streamline_length: float = 300.0,
        runtime=None):
    """Track orientation distribution from a field (__init__.py:217-366).

    ``field`` is a 4D image (the local model inferred from its coefficient
    count) or a prepared field; seeds come from the boundary of ``domain``
    (default: the nonzero voxels of an image field) and the TOD is
    accumulated on the field's image grid (or an image domain's grid for a
    custom field).  Returns 45 normalised SH coefficients per voxel."""
    if not isinstance(n_seeds, (int, __import__("numpy").integer)) or n_seeds < 0:
        raise ValueError("n_seeds must be a non-negative integer.")
    import numpy as np

    if not np.isfinite(maximum_streamline_length) or maximum_streamline_length < 0:
        raise ValueError("maximum_streamline_length must be finite and non-negative.")
    grid_shape = grid_affine = grid_header = None
    domain_image = None
    local_model = None
    if nifti.is_image(field):
        if field.ndim != 4:
            raise ValueError("The tracking image must be four-dimensional.")
        tracking_field = field_module.Image(field)
        domain_image = Nifti1Image(np.any(np.asanyarray(field.dataobj) != 0, axis=-1).astype(np.uint8), field.affine)
        local_model = local.from_shape(field.shape)
        grid_shape, grid_affine = field.shape[:3], field.affine
        grid_header = getattr(field, "header", None)
    elif isinstance(field, field_module.BaseField):
        tracking_field = field
        local_model = local.from_shape((field.n_parameters,)) if algorithm is None else None
        if isinstance(field, field_module.Image):
            grid_affine = np.linalg.inv(field.inverse_affine)
            domain_image = Nifti1Image(np.any(field.values != 0, axis=-1).astype(np.uint8), grid_affine)
            grid_shape = tuple(int(size) for size in field.values.shape[:3])
    else:
        raise TypeError("field must be a Nifti1Image or a BaseField instance.")
    if algorithm is None:
        tracking_algorithm = algorithm_module.Transport(local_model)
    else:
        jobs._validate_algorithm(algorithm)
        tracking_algorithm = algorithm
    if tracking_algorithm.local_model.n_parameters != tracking_field.n_parameters:
        raise ValueError(
            "Algorithm local model parameter count does not match the field: "
            f"{tracking_algorithm.local_model.n_parameters} != {tracking_field.n_parameters}"
        )
    if domain is not None and not (nifti.is_image(domain) or isinstance(domain, domain_module.BaseDomain)):
        raise TypeError("domain must be a BaseDomain, Nifti1Image, or None.")
    tracking_domain = None
    if nifti.is_image(domain):
        if domain.ndim != 3:
            raise ValueError("Domain image must be three-dimensional.")
        domain_image = domain
        if grid_shape is None:
            grid_shape, grid_affine = domain.shape, domain.affine
    elif domain is not None:
        tracking_domain = domain
        if grid_shape is None and isinstance(domain, domain_module.Image):
            grid_shape = tuple(int(size) for size in domain.values.shape)
            grid_affine = np.linalg.inv(domain.inverse_affine)
    elif domain_image is None:
        raise ValueError("A domain is required when the field is not an image field.")
    if grid_shape is None or grid_affine is None:
        raise ValueError("A field image or image-based domain is required to define the TOD grid.")
    image_grid = Nifti1Image(np.zeros(grid_shape, dtype=np.float32), grid_affine, grid_header)
    if tracking_domain is None:
        if not np.any(np.asanyarray(domain_image.dataobj) != 0):
            return Nifti1Image(np.zeros(tuple(grid_shape) + (45,), dtype=np.float32), grid_affine, grid_header)
        tracking_domain = domain_module.Image(domain_image)
    return tracking.tod(tracking_algorithm, tracking_domain, tracking_field, image_grid, n_seeds,
                        maximum_streamline_length=maximum_streamline_length, runtime=runtime)


def write_tractogram(
    filename,
    field,
    seeds,
    domain=None,
    algorithm=None,
    *,
    save_at: float = 1.0,
    maximum_streamline_length: float = 300.0,
    minimum_streamline_length: float = 0.0,
    batch_size: int = 50000,
    seeds_per_pass: int = 1000000,
    runtime=None,
) -> int:
    """Track like :func:`tractogram` and stream the result to ``filename``
    (``.tck`` or ``.trx``, by suffix) without building it in memory; the
    batch writer of tractography/cli/tractogram.py:81-139.  Same arguments,
    validation and results as :func:`tractogram`; returns the number of
    streamlines written."""
    job = jobs.prepare(field, seeds, domain, algorithm, save_at=save_at,
                       maximum_streamline_length=maximum_streamline_length,
                       minimum_streamline_length=minimum_streamline_length, batch_size=batch_size,
                       runtime=runtime)
    if isinstance(job, Tractogram):
        from .streamlines import TckWriter, TrxWriter

        suffix = str(filename).lower().rsplit(".", 1)[-1]
        if suffix not in ("tck", "trx"):
            raise ValueError(f"Unknown tractogram file type: .{suffix}")
        (TckWriter if suffix == "tck" else TrxWriter)(filename).close()
        return 0
    from .runtime import default_runtime

    return jobs.write(job, filename, runtime or default_runtime(), seeds_per_pass)


def tractogram(
    field,
    seeds,
    domain=None,
    algorithm=None,
    *,
    save_at: float = 1.0,
    maximum_streamline_length: float = 300.0,
    minimum_streamline_length: float = 0.0,
    batch_size: int = 50000,
    runtime=None,
) -> Tractogram:
    """Generate streamlines from a 4D image or a prepared field.

    Same contract as the reference's ``tractography.tractogram``
    (tractography/__init__.py:369-540): a 6-coefficient image selects the
    tensor model and a 45-coefficient image spherical harmonics; the default
    algorithm is Transport and the default domain the nonzero voxels of the
    field.  Seeds are split into batches of ``batch_size``; each batch draws
    its own RNG seed from the algorithm, in order, exactly as the
    reference's per-batch calls do, but all batches run in one persistent
    GPU launch.  Streamlines with ``len <= ceil(minimum / save_at)`` points
    are dropped.
    """
    job = jobs.prepare(field, seeds, domain, algorithm, save_at=save_at,
                       maximum_streamline_length=maximum_streamline_length,
                       minimum_streamline_length=minimum_streamline_length, batch_size=batch_size,
                       runtime=runtime)
    if isinstance(job, Tractogram):
        return job
    from .runtime import default_runtime

    return jobs.run(job, runtime or default_runtime())
