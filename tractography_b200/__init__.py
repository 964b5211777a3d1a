"""tractography_b200 -- streamline tracking of cronos-inria/tractography on B200.

A drop-in for the reference's tracking path: the public ``tractogram``
function, the ``algorithm`` (Transport, Diffusion), ``local``
(RealSymmetricSphericalHarmonics, DiffusionTensorImaging), ``field``,
``domain`` and ``seeds`` modules and ``.tck`` output keep the reference's
names, arguments and errors; the OpenCL backend is replaced by compiled
sm_100a CUDA kernels behind the C ABI of ``include/tractography_b200.h``.
"""

from __future__ import annotations

import numpy as np

from . import algorithm as algorithm_module
from . import core, local, nifti, streamlines, tracking
from . import domain as domain_module
from . import field as field_module
from . import seeds
from .algorithm import BaseAlgorithm
from .nifti import Nifti1Image
from .opencl import BufferAccess, OpenCLRuntime
from .runtime import CudaRuntime
from .streamlines import ArraySequence, Tractogram, load_tck, save_tck

algorithm = algorithm_module
domain = domain_module
field = field_module
seeds_module = seeds

__all__ = [
    "ArraySequence", "BufferAccess", "CudaRuntime", "Nifti1Image", "OpenCLRuntime", "Tractogram",
    "algorithm", "core", "domain", "field", "load_tck", "local", "nifti", "save_tck", "seeds",
    "streamlines", "tracking", "tractogram",
]


def _validate_algorithm(tracking_algorithm) -> None:
    if not isinstance(tracking_algorithm, BaseAlgorithm):
        raise TypeError("algorithm must be a BaseAlgorithm instance.")


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

    if nifti.is_image(field):
        if field.ndim != 4:
            raise ValueError("The tracking image must be four-dimensional.")
        tracking_field = field_module.Image(field)
        domain_image = Nifti1Image(np.any(tracking_field.values != 0, axis=-1).astype(np.uint8), field.affine)
        local_model = local.from_shape(field.shape)
    elif isinstance(field, field_module.BaseField):
        tracking_field = field
        local_model = local.from_shape((field.n_parameters,)) if algorithm is None else None
        if isinstance(field, field_module.Image):
            affine = np.linalg.inv(field.inverse_affine)
            domain_image = Nifti1Image(np.any(field.values != 0, axis=-1).astype(np.uint8), affine)
        else:
            domain_image = None
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
    elif domain_image is not None:
        tracking_domain = domain_module.Image(domain_image)
    else:
        raise ValueError(
            "A domain is required when the field is not an image field and "
            "does not provide an image-derived nonzero domain."
        )

    from .runtime import default_runtime

    if isinstance(seeds, (int, np.integer)):
        runtime = runtime or default_runtime()
        seeds = domain_module.seed(tracking_domain, n_seeds, runtime=runtime)
    if len(seeds) == 0:
        return Tractogram([], affine_to_rasmm=np.eye(4))
    runtime = runtime or default_runtime()

    n_steps = tracking._n_steps(save_at, maximum_streamline_length)
    tracking._check_compatible(tracking_algorithm, tracking_field)
    n_batches = (len(seeds) + batch_size - 1) // batch_size
    batch_rng_seeds = [tracking_algorithm.get_rng_seed() for _ in range(n_batches)]
    key = tracking_algorithm.philox_key() if tracking_algorithm.rng_mode() == 1 else 0
    result = tracking.track_packed(tracking_algorithm, tracking_domain, tracking_field, seeds, save_at=save_at,
                                   n_steps=n_steps, batch_size=int(batch_size), batch_rng_seeds=batch_rng_seeds,
                                   runtime=runtime, philox_key=key)
    keep = result.lengths > int(np.ceil(minimum_streamline_length / save_at))
    return Tractogram(result.streamlines(keep), affine_to_rasmm=np.eye(4))
