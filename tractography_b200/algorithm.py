"""Orientation-update algorithms (reference ``tractography/algorithm.py``).

``Transport`` moves the orientation along the gradient of log F on the
sphere; ``Diffusion`` adds tangent-plane Gaussian noise of variance
``noise_variance`` (algorithm.py:56-269).  Both are compiled CUDA code
paths; the NumPy ``update_orientation`` methods are the reference's float64
implementations, and module-level ``update_orientation`` runs on the GPU.

Random streams: by default Diffusion draws from the reference's MWC64X
stream, seeded per tracking call by ``get_rng_seed()`` and per seed by its
index within the call (core.cl:180-245).  ``rng="philox"`` selects a
counter-based Philox4x32-10 stream keyed by (key, global seed index, step),
which does not depend on how seeds are batched.
"""

from __future__ import annotations

import ctypes
from abc import ABC, abstractmethod
from enum import Enum

import numpy as np

from . import _lib
from .core import cart2sph
from .local import BaseLocalModel, model_id


class Algorithm(Enum):
    """Algorithm names (algorithm.py:18-27)."""

    DETERMINISTIC = "deterministic"
    PROBABILISTIC = "probabilistic"
    DIFFUSION = "diffusion"
    TRANSPORT = "transport"

    def __str__(self):
        return self.value


class BaseAlgorithm(ABC):
    """Abstract orientation-update algorithm (algorithm.py:30-53)."""

    algorithm_id: int = -1

    def __init__(self, local_model: BaseLocalModel, step_size: float = 1.0):
        self.local_model = local_model
        self.step_size = step_size

    def get_rng_seed(self) -> int:
        """Seed for per-seed RNG initialisation of one tracking call."""
        return 0

    def rng_mode(self) -> int:
        return _lib.RNG_MWC64X

    def philox_key(self) -> int:
        return 0

    @abstractmethod
    def update_orientation(self, local_models: np.ndarray, orientations: np.ndarray) -> np.ndarray:
        """NumPy implementation."""


class Transport(BaseAlgorithm):
    """Deterministic transport update (algorithm.py:56-156)."""

    algorithm_id = _lib.ALGO_TRANSPORT

    def __init__(self, local_model: BaseLocalModel, step_size: float = 0.001, gamma: float = 1.0):
        super().__init__(local_model, step_size=step_size)
        self.gamma = gamma

    def update_orientation(self, local_models, orientations):
        n = orientations.shape[0]
        mv = self.local_model.evaluate(local_models, orientations)
        phi, theta, _ = cart2sph(*orientations.T)
        sp, cp, st, ct = np.sin(phi), np.cos(phi), np.sin(theta), np.cos(theta)
        et = np.stack([ct * cp, ct * sp, -st], axis=-1)
        ep = np.stack([-sp, cp, np.zeros(n)], axis=-1)
        drift = (mv[:, 1, None] * et + mv[:, 2, None] * ep) / np.maximum(mv[:, 0, None], 1e-6)
        return exps2(orientations, self.step_size * self.gamma * drift, 1.0)


class Diffusion(BaseAlgorithm):
    """Drift plus tangent-plane Gaussian noise (algorithm.py:159-269).

    Args:
        local_model: model giving the value and its angular derivatives.
        step_size: integration time step (also the spatial step).
        gamma: drift and noise scale.
        noise_variance: variance of the tangent-plane noise.
        seed: seed of the generator that draws one stream seed per call.
        rng: ``"mwc64x"`` (reference stream, default) or ``"philox"``.
    """

    algorithm_id = _lib.ALGO_DIFFUSION

    def __init__(self, local_model: BaseLocalModel, step_size: float = 0.001, gamma: float = 1.0,
                 noise_variance: float = 0.1, seed: int | None = None, rng: str = "mwc64x"):
        super().__init__(local_model, step_size=step_size)
        self.gamma = gamma
        self.noise_variance = noise_variance
        self._rng = np.random.default_rng(seed)
        if rng not in ("mwc64x", "philox"):
            raise ValueError("rng must be 'mwc64x' or 'philox'")
        self.rng = rng

    def get_rng_seed(self) -> int:
        """Draw one seed; each seed's stream is derived from it (algorithm.py:239-241)."""
        return int(self._rng.integers(0, np.iinfo(np.uint32).max, dtype=np.uint32))

    def rng_mode(self) -> int:
        return _lib.RNG_PHILOX if self.rng == "philox" else _lib.RNG_MWC64X

    def philox_key(self) -> int:
        return int(self._rng.integers(0, 2 ** 63 - 1, dtype=np.int64))

    def update_orientation(self, local_models, orientations):
        n = orientations.shape[0]
        mv = self.local_model.evaluate(local_models, orientations)
        phi, theta, _ = cart2sph(*orientations.T)
        sp, cp, st, ct = np.sin(phi), np.cos(phi), np.sin(theta), np.cos(theta)
        et = np.stack([ct * cp, ct * sp, -st], axis=-1)
        ep = np.stack([-sp, cp, np.zeros(n)], axis=-1)
        drift = (mv[:, 1, None] * et + mv[:, 2, None] * ep) / np.maximum(mv[:, 0, None], 1e-6)
        noise = np.zeros_like(drift)
        if self.noise_variance > 0.0:
            samples = self._rng.standard_normal((n, 2))
            noise = samples[:, :1] * et + samples[:, 1:] * ep
        tangent = self.gamma * self.step_size * drift + np.sqrt(
            self.noise_variance * self.gamma * self.step_size) * noise
        return exps2(orientations, tangent, 1.0)


def exps2(p: np.ndarray, x: np.ndarray, t: float) -> np.ndarray:
    """Spherical exponential map of tangent vectors x at points p (algorithm.py:680-698)."""
    n = np.linalg.norm(x, axis=1)
    c = np.cos(t * n)
    s = np.sin(t * n)
    scaled_sine = np.divide(s, n, out=np.zeros_like(n), where=n != 0)
    return c[:, np.newaxis] * p + x * scaled_sine[:, np.newaxis]


def algorithm_id(algorithm: BaseAlgorithm) -> int:
    if isinstance(algorithm, Transport):
        return _lib.ALGO_TRANSPORT
    if isinstance(algorithm, Diffusion):
        return _lib.ALGO_DIFFUSION
    raise NotImplementedError(
        f"{type(algorithm).__name__} has no compiled CUDA code path; only Transport and Diffusion "
        "are supported"
    )


def to_struct(algorithm: BaseAlgorithm, rng_seed: int = 0, philox_key: int = 0,
              seed_offset: int = 0) -> _lib.Algorithm:
    """The ``tg_algorithm`` of an algorithm object for one call."""
    a = _lib.Algorithm()
    a.algorithm = algorithm_id(algorithm)
    a.step_size = float(algorithm.step_size)
    a.gamma = float(algorithm.gamma)
    a.noise_variance = float(getattr(algorithm, "noise_variance", 0.0))
    a.rng_mode = algorithm.rng_mode()
    a.rng_seed = int(rng_seed) & 0xFFFFFFFF
    a.philox_key = int(philox_key) & 0xFFFFFFFFFFFFFFFF
    a.seed_offset = int(seed_offset)
    return a


def update_orientation(algorithm: BaseAlgorithm, local_models, orientations, runtime=None) -> np.ndarray:
    """One GPU orientation update per row (algorithm.py:701-790)."""
    orientations = np.asarray(orientations)
    n = orientations.shape[0]
    if n == 0:
        return np.empty((0, 3), dtype=np.float32)
    local_models = np.asarray(local_models)
    C = algorithm.local_model.n_parameters
    if local_models.ndim != 2 or local_models.shape[1] != C or local_models.shape[0] != n:
        raise ValueError(f"Expected local_models to have shape ({n}, {C}), but got {local_models.shape}")
    from .runtime import default_runtime

    runtime = runtime or default_runtime()
    import torch

    mid = model_id(algorithm.local_model)
    a = to_struct(algorithm, rng_seed=algorithm.get_rng_seed(),
                  philox_key=algorithm.philox_key() if algorithm.rng_mode() == _lib.RNG_PHILOX else 0)
    o4 = np.zeros((n, 4), dtype=np.float32)
    o4[:, :3] = orientations
    with runtime.device_scope():
        d_params = runtime.to_device(np.ascontiguousarray(local_models, dtype=np.float32))
        d_o = runtime.to_device(o4)
        d_out = runtime.empty((n, 4), torch.float32)
        _lib.check(runtime.lib.tg_update_orientation(mid, C, ctypes.byref(a), ctypes.c_void_p(d_params.data_ptr()),
                                                     ctypes.c_void_p(d_o.data_ptr()), n,
                                                     ctypes.c_void_p(d_out.data_ptr()),
                                                     ctypes.c_void_p(runtime.stream_handle)))
        return d_out.cpu().numpy()[:, :3].copy()
