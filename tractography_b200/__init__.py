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
from . import core, jobs, local, nifti, streamlines, tracking
from . import domain as domain_module
from . import field as field_module
from . import seeds
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
    "algorithm", "core", "domain", "field", "jobs", "load_tck", "local", "nifti", "save_tck", "seeds",
    "streamlines", "tracking", "tractogram",
]


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
