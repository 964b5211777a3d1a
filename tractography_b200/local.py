"""Local models: spherical harmonics and diffusion tensors.

Reference: ``tractography/local.py``.  In the reference each model returns an
OpenCL source fragment that the tracker compiles; here the models are
identifiers of compiled CUDA code paths (``model_id``), plus the same
float64 NumPy ``evaluate`` methods the reference keeps as implementation
references.  ``evaluate()`` at module level runs on the GPU.
"""

from __future__ import annotations

import ctypes
from abc import ABC, abstractmethod
from collections.abc import Sequence

import numpy as np

from . import _lib
from .core import cart2sph, ishtmtx

SOFTMAX_SCALE = 100.0   # local.py:17
MAX_SH_COEFFICIENTS = 45


class BaseLocalModel(ABC):
    """A model evaluated at orientations (local.py:20-71).

    ``evaluate`` returns (n, 3): value, d/dtheta and (d/dphi)/sin(theta).
    """

    model_id: int = -1
    opencl_model: str = ""

    def __init__(self, n_parameters: int):
        self.n_parameters = n_parameters

    @abstractmethod
    def evaluate(self, parameters: np.ndarray, orientations: np.ndarray) -> np.ndarray:
        """Evaluate with NumPy (float64 reference implementation)."""


class RealSymmetricSphericalHarmonics(BaseLocalModel):
    """Real symmetric SH model (MRtrix basis) with a softplus output.

    Supports 1 to 45 coefficients (degree <= 8); coefficients beyond
    ``n_parameters`` in the last band are treated as zero, as the reference's
    loop over the first ``n_parameters`` terms does (local.py:106).
    """

    model_id = _lib.MODEL_SH
    opencl_model = "MODEL_SYMMETRIC_REAL_SPHERICAL_HARMONICS"

    def evaluate(self, parameters, orientations):
        """NumPy reference of local.py:123-189."""
        orientations = np.asarray(orientations)
        if orientations.shape[0] == 0:
            return np.empty((0, 3), dtype=np.float32)
        parameters = np.asarray(parameters)

        def softmax(x, k):
            with np.errstate(over="ignore"):
                return np.where(x * k < 30.0, np.log(1 + np.exp(k * x)) / k, x)

        def dsoftmax(x, k):
            with np.errstate(over="ignore"):
                return 1.0 / (1 + np.exp(-k * x))

        phi, theta, _ = cart2sph(*orientations.T)
        mtx, der = ishtmtx(phi, theta, self.n_parameters)
        value = np.einsum("ij,ij->i", mtx, parameters)
        d = dsoftmax(value, SOFTMAX_SCALE)
        value = softmax(value, SOFTMAX_SCALE)
        dphi_numerator = np.einsum("ij,ij->i", der[1], parameters)
        sin_theta = np.sin(theta)
        at_pole = np.isclose(sin_theta, 0.0, atol=1e-7, rtol=0.0)
        dphi = np.divide(dphi_numerator, sin_theta, out=np.zeros_like(dphi_numerator), where=~at_pole)
        dtheta = np.einsum("ij,ij->i", der[0], parameters)
        if np.any(at_pole):
            # Pole limits evaluated just inside the valid range.
            pole_theta = np.where(np.cos(theta[at_pole]) >= 0, 1e-6, np.pi - 1e-6)
            _, pole_der = ishtmtx(phi[at_pole], pole_theta, self.n_parameters)
            pp = parameters[at_pole]
            dtheta[at_pole] = np.einsum("ij,ij->i", pole_der[0], pp)
            dphi[at_pole] = np.einsum("ij,ij->i", pole_der[1], pp) / np.sin(pole_theta)
        return np.stack([value, dtheta * d, dphi * d], axis=-1)


class DiffusionTensorImaging(BaseLocalModel):
    """Tensor model u^T D u with (Dxx, Dyy, Dzz, Dxy, Dxz, Dyz) coefficients."""

    model_id = _lib.MODEL_DTI
    opencl_model = "MODEL_DTI"

    def __init__(self):
        super().__init__(6)

    def evaluate(self, parameters, orientations):
        """NumPy reference of local.py:233-262."""
        orientations = np.asarray(orientations)
        n = orientations.shape[0]
        if n == 0:
            return np.empty((0, 3), dtype=np.float32)
        parameters = np.asarray(parameters)
        tensor = np.zeros((n, 3, 3), dtype=np.result_type(parameters, orientations))
        tensor[:, 0, 0] = parameters[:, 0]
        tensor[:, 1, 1] = parameters[:, 1]
        tensor[:, 2, 2] = parameters[:, 2]
        tensor[:, 0, 1] = tensor[:, 1, 0] = parameters[:, 3]
        tensor[:, 0, 2] = tensor[:, 2, 0] = parameters[:, 4]
        tensor[:, 1, 2] = tensor[:, 2, 1] = parameters[:, 5]
        du = np.einsum("nij,nj->ni", tensor, orientations)
        value = np.einsum("ni,ni->n", orientations, du)
        phi, theta, _ = cart2sph(*orientations.T)
        st, ct = np.sin(theta), np.cos(theta)
        sp, cp = np.sin(phi), np.cos(phi)
        e_theta = np.stack([ct * cp, ct * sp, -st], axis=-1)
        e_phi = np.stack([-sp, cp, np.zeros(n)], axis=-1)
        dtheta = 2.0 * np.einsum("ni,ni->n", du, e_theta)
        dphi = 2.0 * np.einsum("ni,ni->n", du, e_phi)
        return np.stack([value, dtheta, dphi], axis=-1).astype(np.float32)


def from_shape(shape: Sequence[int]) -> BaseLocalModel:
    """Local model for a field's coefficient count (local.py:265-282)."""
    if len(shape) == 0:
        raise ValueError("A local-model shape must include a coefficient dimension.")
    n_parameters = shape[-1]
    if n_parameters == 6:
        return DiffusionTensorImaging()
    if n_parameters == 45:
        return RealSymmetricSphericalHarmonics(n_parameters)
    raise ValueError("For now, only DTI and fODF with 45 coefficients are supported (lmax=8).")


def model_id(model: BaseLocalModel) -> int:
    """Compiled code path of a model; custom subclasses have none."""
    if isinstance(model, DiffusionTensorImaging):
        return _lib.MODEL_DTI
    if isinstance(model, RealSymmetricSphericalHarmonics):
        if not 1 <= model.n_parameters <= MAX_SH_COEFFICIENTS:
            raise NotImplementedError(
                f"spherical-harmonic models support 1 to {MAX_SH_COEFFICIENTS} coefficients, "
                f"got {model.n_parameters}"
            )
        return _lib.MODEL_SH
    raise NotImplementedError(
        f"{type(model).__name__} has no compiled CUDA code path; only "
        "RealSymmetricSphericalHarmonics and DiffusionTensorImaging are supported"
    )


def evaluate(model: BaseLocalModel, parameters, orientations, runtime=None) -> np.ndarray:
    """Evaluate a model on the GPU (local.py:285-363).

    Returns (n, 3) float32: value, d/dtheta and (d/dphi)/sin(theta).
    """
    orientations = np.asarray(orientations)
    n = orientations.shape[0]
    if n == 0:
        return np.empty((0, 3), dtype=np.float32)
    from .runtime import default_runtime

    runtime = runtime or default_runtime()
    mid = model_id(model)
    params = np.ascontiguousarray(parameters, dtype=np.float32)
    if params.shape != (n, model.n_parameters):
        raise ValueError(f"Expected parameters of shape ({n}, {model.n_parameters}), but got {params.shape}")
    o4 = np.zeros((n, 4), dtype=np.float32)
    o4[:, :3] = orientations
    import torch

    with runtime.device_scope():
        d_params = runtime.to_device(params)
        d_o = runtime.to_device(o4)
        d_out = runtime.empty((n, 3), torch.float32)
        _lib.check(runtime.lib.tg_local_evaluate(mid, model.n_parameters, ctypes.c_void_p(d_params.data_ptr()),
                                                 ctypes.c_void_p(d_o.data_ptr()), n,
                                                 ctypes.c_void_p(d_out.data_ptr()),
                                                 ctypes.c_void_p(runtime.stream_handle)))
        out = d_out.cpu()
    return out.numpy()
