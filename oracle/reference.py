"""ctypes access to oracle/_ref/libtgref.so: the reference's kernels run on the CPU.

Test infrastructure only (tests, smoke check, benchmark CPU legs).  The
library is built by oracle/build_ref.py from the reference sources; it is
absent where the reference tree is not available, and callers must check
``available()``.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "_ref" / "libtgref.so"
_lib = None


def available() -> bool:
    return LIB_PATH.exists()


def lib():
    global _lib
    if _lib is None:
        _lib = ctypes.CDLL(str(LIB_PATH))
    return _lib


def _variant(model: str, n_coefficients: int, algorithm: str) -> str:
    if model == "dti":
        return f"dti_{algorithm}"
    return f"sh{n_coefficients}_{algorithm}"


def tractogram_raw(mask, mask_inv_affine, field, field_inv_affine, model, algorithm, step_size, gamma,
                   noise_variance, rng_seed, seeds, save_at, n_steps, threads=1):
    """Run the reference kernel; returns (dense (n, n_steps, 4) points, lengths, accepted steps)."""
    field = np.ascontiguousarray(field, dtype=np.float32)
    mask = np.ascontiguousarray(np.asarray(mask) != 0, dtype=np.int32)
    seeds = np.ascontiguousarray(seeds, dtype=np.float32)
    minv = np.ascontiguousarray(mask_inv_affine, dtype=np.float32)
    finv = np.ascontiguousarray(field_inv_affine, dtype=np.float32)
    mdims = np.array(mask.shape, dtype=np.uint32)
    fdims = np.array(field.shape, dtype=np.uint32)
    n = len(seeds)
    out = np.zeros((n, n_steps, 4), np.float32)
    lengths = np.zeros(n, np.uint32)
    fn = getattr(lib(), "tgref_" + _variant(model, field.shape[3], algorithm))
    fn.restype = ctypes.c_ulonglong
    P = ctypes.c_void_p
    fn.argtypes = [P, P, P, P, P, P, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_uint, P,
                   ctypes.c_uint, P, P, ctypes.c_float, ctypes.c_uint, ctypes.c_int]
    steps = fn(mask.ctypes.data, mdims.ctypes.data, minv.ctypes.data, field.ctypes.data, fdims.ctypes.data,
               finv.ctypes.data, step_size, gamma, noise_variance, rng_seed & 0xFFFFFFFF, seeds.ctypes.data, n,
               out.ctypes.data, lengths.ctypes.data, save_at, n_steps, threads)
    return out, lengths, int(steps)


def tractogram(domain, field, algorithm, seeds, rng_seed, save_at, n_steps, threads=1):
    """Same as tractogram_raw for package domain/field/algorithm objects."""
    model = "dti" if algorithm.local_model.n_parameters == 6 and type(algorithm.local_model).__name__ == \
        "DiffusionTensorImaging" else "sh"
    kind = "diffusion" if hasattr(algorithm, "noise_variance") else "transport"
    return tractogram_raw(domain.values, domain.inverse_affine, field.values, field.inverse_affine, model, kind,
                          algorithm.step_size, algorithm.gamma, getattr(algorithm, "noise_variance", 0.0),
                          rng_seed, seeds, save_at, n_steps, threads)


def tractogram_steps(domain, field, kind, step_size, gamma, noise_variance, seeds, rng_seed, save_at, n_steps,
                     threads):
    """Accepted steps of a reference-kernel run (for timing)."""
    model = "sh" if field.values.shape[3] != 6 else "dti"
    return tractogram_raw(domain.values, domain.inverse_affine, field.values, field.inverse_affine, model, kind,
                          step_size, gamma, noise_variance, rng_seed, seeds, save_at, n_steps, threads)[2]


def update_orientation(model, n_coefficients, algorithm, step_size, gamma, noise_variance, rng_seed, params,
                       orientations):
    """The reference's standalone orientation-update kernel, one row per orientation."""
    params = np.ascontiguousarray(params, dtype=np.float32)
    o4 = np.zeros((len(orientations), 4), np.float32)
    o4[:, :3] = orientations
    out = np.zeros_like(o4)
    fn = getattr(lib(), "tgref_update_u_" + _variant(model, n_coefficients, algorithm))
    P = ctypes.c_void_p
    fn.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_uint, P, P, ctypes.c_uint, P]
    fn(step_size, gamma, noise_variance, rng_seed & 0xFFFFFFFF, params.ctypes.data, o4.ctypes.data, len(o4),
       out.ctypes.data)
    return out[:, :3]


def bvh_hits(vertices4, triangles4, bounds_min, bounds_max, nodes, ordered, starts, ends):
    """The reference's bvh_segment_hit (utils/bvh.cl:83-131) per segment.

    Returns (found, triangle, (n, 4) barycentric xyz + t)."""
    arrays = [np.ascontiguousarray(a, dt) for a, dt in ((vertices4, np.float32), (triangles4, np.uint32),
                                                        (bounds_min, np.float32), (bounds_max, np.float32),
                                                        (nodes, np.int32), (ordered, np.uint32))]
    s4 = np.zeros((len(starts), 4), np.float32)
    e4 = np.zeros((len(ends), 4), np.float32)
    s4[:, :3], e4[:, :3] = np.asarray(starts)[:, :3], np.asarray(ends)[:, :3]
    n = len(s4)
    found = np.zeros(n, np.uint8)
    tri = np.zeros(n, np.uint32)
    hit = np.zeros((n, 4), np.float32)
    fn = lib().tgref_bvh_hits
    P = ctypes.c_void_p
    fn.argtypes = [P] * 6 + [ctypes.c_uint, P, P, ctypes.c_uint, P, P, P]
    fn(*[a.ctypes.data for a in arrays], len(arrays[4]), s4.ctypes.data, e4.ctypes.data, n, found.ctypes.data,
       tri.ctypes.data, hit.ctypes.data)
    return found.astype(bool), tri, hit


def boundary_seeds(vertices4, triangles4, cumulative, rng_seed, n):
    """The reference's boundary sampler (domain.py:95-120 via domain.seed): (n, 8) seeds."""
    v = np.ascontiguousarray(vertices4, np.float32)
    t = np.ascontiguousarray(triangles4, np.uint32)
    c = np.ascontiguousarray(cumulative, np.float32)
    loc = np.zeros((n, 4), np.float32)
    ori = np.zeros((n, 4), np.float32)
    fn = lib().tgref_boundary_seeds
    P = ctypes.c_void_p
    fn.argtypes = [P, P, P, ctypes.c_uint, ctypes.c_uint, ctypes.c_uint, P, P]
    fn(v.ctypes.data, t.ctypes.data, c.ctypes.data, len(c), rng_seed & 0xFFFFFFFF, n, loc.ctypes.data,
       ori.ctypes.data)
    return np.hstack((loc, ori))


def _domain_arrays(domain, bvh):
    boundary = domain.boundary_arrays()
    mask = np.ascontiguousarray(np.asarray(domain.values) != 0, dtype=np.int32)
    arrays = [*boundary, bvh.bounds_min, bvh.bounds_max, bvh.nodes, bvh.ordered, mask,
              np.array(mask.shape, np.uint32), np.ascontiguousarray(domain.inverse_affine, np.float32)]
    return arrays, len(boundary[2]), len(bvh.nodes)


def _product(kind, algorithm_kind, domain, field, bvh, step, gamma, noise, rng_seed, n_seeds, n_steps, tail, threads):
    fld = np.ascontiguousarray(field.values, np.float32)
    arrays, n_tri, n_nodes = _domain_arrays(domain, bvh)
    fdims = np.array(fld.shape, np.uint32)
    finv = np.ascontiguousarray(field.inverse_affine, np.float32)
    fn = getattr(lib(), f"tgref_{kind}_sh45_{algorithm_kind}")
    P, U, F = ctypes.c_void_p, ctypes.c_uint, ctypes.c_float
    v, t, c, bmin, bmax, nodes, ordered, mask, mdims, minv = arrays
    args = [v.ctypes.data, t.ctypes.data, c.ctypes.data, n_tri, bmin.ctypes.data, bmax.ctypes.data, nodes.ctypes.data,
            ordered.ctypes.data, n_nodes, mask.ctypes.data, mdims.ctypes.data, minv.ctypes.data, fld.ctypes.data,
            fdims.ctypes.data, finv.ctypes.data, step, gamma, noise, rng_seed & 0xFFFFFFFF, n_seeds, n_steps]
    types = [P, P, P, U, P, P, P, P, U, P, P, P, P, P, P, F, F, F, U, U, U]
    return fn, args, types, (fld, arrays, fdims, finv)


def tod(domain, field, bvh, algorithm_kind, step, gamma, noise, rng_seed, n_seeds, n_steps, out_shape, out_inverse,
        threads=1):
    """The reference's `tod` kernel (SH lmax 8, image domain): raw (X, Y, Z, 45) coefficients."""
    fn, args, types, keep = _product("tod", algorithm_kind, domain, field, bvh, step, gamma, noise, rng_seed, n_seeds,
                                     n_steps, None, threads)
    odims = np.array(out_shape, np.uint32)
    oinv = np.ascontiguousarray(out_inverse, np.float32)
    out = np.zeros(tuple(out_shape) + (45,), np.float32)
    fn.argtypes = types + [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    fn(*args, odims.ctypes.data, oinv.ctypes.data, out.ctypes.data, threads)
    return out


def connectome(domain, field, bvh, algorithm_kind, step, gamma, noise, rng_seed, n_seeds, n_steps, minimum_length,
               threads=1):
    """The reference's `connectome` kernel (SH lmax 8, image domain): rows, columns, weights (9 per seed)."""
    fn, args, types, keep = _product("connectome", algorithm_kind, domain, field, bvh, step, gamma, noise, rng_seed,
                                     n_seeds, n_steps, None, threads)
    rows = np.empty(9 * n_seeds, np.int32)
    cols = np.zeros(9 * n_seeds, np.int32)
    w = np.zeros(9 * n_seeds, np.float32)
    fn.argtypes = types + [ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    fn(*args, minimum_length, rows.ctypes.data, cols.ctypes.data, w.ctypes.data, threads)
    return rows, cols, w


def seeds_from_fod(model, fod_sparse, voxels, affine, states, threads=1):
    """The reference's FOD seeding kernel (utils/seeds.cl:99-118 as seeds.py:174-216
    builds it) on the CPU: sparse (nnz, C) coefficients, (nnz, 4) voxel indices,
    the float32 voxel-to-world affine and (n, 2) MWC64X states.  Returns the
    (n, 8) seeds and the states after the draws."""
    C = 6 if model == "dti" else 45
    fod_sparse = np.ascontiguousarray(fod_sparse, dtype=np.float32)
    assert fod_sparse.shape[1] == C
    voxels = np.ascontiguousarray(voxels, dtype=np.float32)
    affine = np.ascontiguousarray(affine, dtype=np.float32)
    states = np.array(states, dtype=np.uint32, order="C", copy=True)
    n = states.shape[0]
    seeds = np.zeros((n, 8), np.float32)
    fn = getattr(lib(), "tgref_fodseed_" + ("dti" if model == "dti" else "sh45"))
    P = ctypes.c_void_p
    fn.argtypes = [P, P, P, P, P, ctypes.c_uint, ctypes.c_uint, ctypes.c_int]
    fn.restype = None
    fn(fod_sparse.ctypes.data, voxels.ctypes.data, affine.ctypes.data, states.ctypes.data, seeds.ctypes.data,
       len(voxels), n, threads)
    return seeds, states
