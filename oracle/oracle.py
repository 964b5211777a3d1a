"""ctypes bindings for the CPU oracle (test infrastructure only).

The oracle restates the reference's tracking path in plain C
(``oracle/tg_oracle.c``).  Only the tests, the smoke check and the
benchmark's CPU-baseline leg import this module; the product never does.
"""

from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libtgoracle.so"

MODEL_SH, MODEL_DTI = 0, 1
ALGO_TRANSPORT, ALGO_DIFFUSION = 0, 1
RNG_MWC64X, RNG_PHILOX = 0, 1


class Problem(ctypes.Structure):
    _fields_ = [
        ("mask", ctypes.c_void_p),
        ("mask_dims", ctypes.c_uint32 * 3),
        ("mask_inv_affine", ctypes.c_float * 16),
        ("field", ctypes.c_void_p),
        ("field_dims", ctypes.c_uint32 * 4),
        ("field_inv_affine", ctypes.c_float * 16),
        ("model", ctypes.c_int32),
        ("algorithm", ctypes.c_int32),
        ("step_size", ctypes.c_float),
        ("gamma", ctypes.c_float),
        ("noise_variance", ctypes.c_float),
        ("rng_mode", ctypes.c_int32),
        ("rng_seed", ctypes.c_uint32),
        ("philox_key", ctypes.c_uint64),
        ("seed_offset", ctypes.c_uint64),
        ("save_at", ctypes.c_float),
        ("n_steps", ctypes.c_uint32),
    ]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        _lib = ctypes.CDLL(str(LIB_PATH))
        P = ctypes.c_void_p
        U32, I32, F = ctypes.c_uint32, ctypes.c_int32, ctypes.c_float
        _lib.tgo_tractogram.argtypes = [P, P, U32, P, P, ctypes.c_int]
        _lib.tgo_tractogram.restype = ctypes.c_uint64
        _lib.tgo_contains.argtypes = [P, P, U32, P]
        _lib.tgo_field_evaluate.argtypes = [P, P, U32, P]
        _lib.tgo_local_evaluate.argtypes = [I32, U32, P, P, U32, P]
        _lib.tgo_update_orientation.argtypes = [P, U32, P, P, U32, P]
        _lib.tgo_seeds_from_fod.argtypes = [I32, U32, P, P, U32, P, P, U32, P, ctypes.c_int]
        _lib.tgo_rng_init.argtypes = [U32, U32, P]
        _lib.tgo_randu_stream.argtypes = [U32, U32, U32, P]
        _lib.tgo_randn_stream.argtypes = [U32, U32, U32, P]
        _lib.tgo_randi_stream.argtypes = [U32, U32, U32, U32, P]
        _lib.tgo_philox.argtypes = [P, P, P]
        _lib.tgo_math.argtypes = [ctypes.c_int, P, U32, P]
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class Case:
    """Holds the arrays of one problem so their memory outlives the call."""

    def __init__(self, *, mask=None, mask_inv_affine=None, field=None, field_inv_affine=None,
                 model=MODEL_SH, algorithm=ALGO_TRANSPORT, step_size=0.001, gamma=1.0,
                 noise_variance=0.0, rng_mode=RNG_MWC64X, rng_seed=0, philox_key=0,
                 seed_offset=0, save_at=1.0, n_steps=0):
        self.p = Problem()
        if mask is not None:
            self.mask = np.ascontiguousarray(mask != 0, dtype=np.int32)
            self.p.mask = self.mask.ctypes.data
            self.p.mask_dims[:] = list(self.mask.shape)
            self.p.mask_inv_affine[:] = list(np.asarray(mask_inv_affine, np.float32).ravel())
        if field is not None:
            self.field = np.ascontiguousarray(field, dtype=np.float32)
            self.p.field = self.field.ctypes.data
            self.p.field_dims[:] = list(self.field.shape)
            self.p.field_inv_affine[:] = list(np.asarray(field_inv_affine, np.float32).ravel())
        self.p.model = model
        self.p.algorithm = algorithm
        self.p.step_size = step_size
        self.p.gamma = gamma
        self.p.noise_variance = noise_variance
        self.p.rng_mode = rng_mode
        self.p.rng_seed = rng_seed & 0xFFFFFFFF
        self.p.philox_key = philox_key
        self.p.seed_offset = seed_offset
        self.p.save_at = save_at
        self.p.n_steps = n_steps

    def tractogram(self, seeds, n_threads=1, return_steps=False):
        seeds = np.ascontiguousarray(seeds, dtype=np.float32)
        n = seeds.shape[0]
        out = np.zeros((n, self.p.n_steps, 4), dtype=np.float32)
        lengths = np.zeros(n, dtype=np.uint32)
        steps = lib().tgo_tractogram(ctypes.byref(self.p), _ptr(seeds), n, _ptr(out), _ptr(lengths), n_threads)
        if return_steps:
            return out, lengths, int(steps)
        return out, lengths

    def contains(self, points):
        pts = _points4(points)
        out = np.zeros(len(pts), dtype=np.uint8)
        lib().tgo_contains(ctypes.byref(self.p), _ptr(pts), len(pts), _ptr(out))
        return out.astype(bool)

    def field_evaluate(self, points):
        pts = _points4(points)
        out = np.zeros((len(pts), self.p.field_dims[3]), dtype=np.float32)
        lib().tgo_field_evaluate(ctypes.byref(self.p), _ptr(pts), len(pts), _ptr(out))
        return out

    def update_orientation(self, params, orientations):
        params = np.ascontiguousarray(params, dtype=np.float32)
        o = _points4(orientations, w=0.0)
        out = np.zeros((len(o), 4), dtype=np.float32)
        lib().tgo_update_orientation(ctypes.byref(self.p), params.shape[1], _ptr(params), _ptr(o), len(o), _ptr(out))
        return out[:, :3]


def _points4(points, w=1.0):
    points = np.asarray(points, dtype=np.float32).reshape(-1, points.shape[-1] if np.ndim(points) > 1 else 3)
    out = np.full((len(points), 4), w, dtype=np.float32)
    out[:, :3] = points[:, :3]
    return out


def local_evaluate(model, params, orientations):
    params = np.ascontiguousarray(params, dtype=np.float32)
    o = _points4(orientations, w=0.0)
    out = np.zeros((len(o), 3), dtype=np.float32)
    lib().tgo_local_evaluate(model, params.shape[1], _ptr(params), _ptr(o), len(o), _ptr(out))
    return out


def seeds_from_fod(model, fod_sparse, voxels, affine, states, n_threads=1):
    fod_sparse = np.ascontiguousarray(fod_sparse, dtype=np.float32)
    voxels = np.ascontiguousarray(voxels, dtype=np.float32)
    affine = np.ascontiguousarray(affine, dtype=np.float32)
    states = np.ascontiguousarray(states, dtype=np.uint32)
    n = states.shape[0]
    out = np.zeros((n, 8), dtype=np.float32)
    lib().tgo_seeds_from_fod(model, fod_sparse.shape[1], _ptr(fod_sparse), _ptr(voxels), len(voxels),
                             _ptr(affine), _ptr(states), n, _ptr(out), n_threads)
    return out


def rng_init(seed, stream_id):
    out = np.zeros(2, dtype=np.uint32)
    lib().tgo_rng_init(seed & 0xFFFFFFFF, stream_id & 0xFFFFFFFF, _ptr(out))
    return out


def randu_stream(state, n):
    out = np.zeros(n, dtype=np.float32)
    lib().tgo_randu_stream(int(state[0]), int(state[1]), n, _ptr(out))
    return out


def randn_stream(state, n):
    out = np.zeros(n, dtype=np.float32)
    lib().tgo_randn_stream(int(state[0]), int(state[1]), n, _ptr(out))
    return out


def randi_stream(state, n, maximum):
    out = np.zeros(n, dtype=np.uint32)
    lib().tgo_randi_stream(int(state[0]), int(state[1]), n, maximum, _ptr(out))
    return out


def philox(counter, key):
    c = np.ascontiguousarray(counter, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    lib().tgo_philox(_ptr(c), _ptr(k), _ptr(out))
    return out


def math(which, x):
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.zeros_like(x)
    code = {"sin": 0, "cos": 1, "exp": 2, "log": 3}[which]
    lib().tgo_math(code, _ptr(x), x.size, _ptr(out))
    return out
