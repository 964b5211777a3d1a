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
        ("mesh", ctypes.c_void_p),
    ]


class Bvh(ctypes.Structure):
    _fields_ = [
        ("vertices", ctypes.c_void_p),
        ("triangles", ctypes.c_void_p),
        ("bounds_min", ctypes.c_void_p),
        ("bounds_max", ctypes.c_void_p),
        ("nodes", ctypes.c_void_p),
        ("ordered_triangles", ctypes.c_void_p),
        ("n_nodes", ctypes.c_uint32),
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
        _lib.tgo_tractogram_ids.argtypes = [P, P, P, U32, P, P, ctypes.c_int]
        _lib.tgo_tractogram_ids.restype = ctypes.c_uint64
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
        _lib.tgo_segment_hits.argtypes = [P, P, P, U32, P, P, P, ctypes.c_int]
        _lib.tgo_boundary_seeds.argtypes = [P, P, P, U32, U32, U32, P]
        _lib.tgo_tod.argtypes = [P, P, P, P, U32, U32, U32, P, P, P]
        _lib.tgo_connectome.argtypes = [P, P, P, P, P, U32, U32, U32, F, P, P, P]
        _lib.tgo_mesh_contains.argtypes = [P, F, F, F]
        _lib.tgo_mesh_contains.restype = ctypes.c_int
        _lib.tgo_bvh_count_hits.argtypes = [P, P, P]
        _lib.tgo_bvh_count_hits.restype = U32
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class Case:
    """Holds the arrays of one problem so their memory outlives the call."""

    def __init__(self, *, mask=None, mask_inv_affine=None, field=None, field_inv_affine=None,
                 model=MODEL_SH, algorithm=ALGO_TRANSPORT, step_size=0.001, gamma=1.0,
                 noise_variance=0.0, rng_mode=RNG_MWC64X, rng_seed=0, philox_key=0,
                 seed_offset=0, save_at=1.0, n_steps=0, mesh=None):
        self.p = Problem()
        if mesh is not None:
            self.mesh = mesh
            self.p.mesh = ctypes.addressof(mesh.struct)
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

    def tractogram_ids(self, seeds, ids, n_threads=1, return_steps=False):
        """Seeds taken out of a larger call: seed k is work item ids[k] of it."""
        seeds = np.ascontiguousarray(seeds, dtype=np.float32)
        ids = np.ascontiguousarray(ids, dtype=np.uint32)
        n = seeds.shape[0]
        assert ids.shape == (n,)
        out = np.zeros((n, self.p.n_steps, 4), dtype=np.float32)
        lengths = np.zeros(n, dtype=np.uint32)
        steps = lib().tgo_tractogram_ids(ctypes.byref(self.p), _ptr(seeds), _ptr(ids), n, _ptr(out), _ptr(lengths),
                                         n_threads)
        if return_steps:
            return out, lengths, int(steps)
        return out, lengths

    def tod(self, boundary, n_seeds, n_steps, out_shape, out_inverse_affine):
        """tracking.py:181-385 raw (un-normalised) TOD coefficients (X, Y, Z, 45)."""
        v, t, c = (np.ascontiguousarray(a, dt) for a, dt in zip(boundary, (np.float32, np.uint32, np.float32)))
        dims = np.ascontiguousarray(out_shape, dtype=np.uint32)
        inv = np.ascontiguousarray(out_inverse_affine, dtype=np.float32)
        out = np.zeros(tuple(int(x) for x in out_shape) + (45,), np.float32)
        lib().tgo_tod(ctypes.byref(self.p), _ptr(v), _ptr(t), _ptr(c), len(c), n_seeds, n_steps, _ptr(dims),
                      _ptr(inv), _ptr(out))
        return out

    def connectome(self, boundary_bvh, boundary, n_seeds, n_steps, minimum_length=0.0):
        """tracking.py:388-602 contributions: rows, columns, weights (9 per seed)."""
        v, t, c = (np.ascontiguousarray(a, dt) for a, dt in zip(boundary, (np.float32, np.uint32, np.float32)))
        rows = np.empty(9 * n_seeds, np.int32)
        cols = np.zeros(9 * n_seeds, np.int32)
        w = np.zeros(9 * n_seeds, np.float32)
        lib().tgo_connectome(ctypes.byref(self.p), ctypes.byref(boundary_bvh.struct), _ptr(v), _ptr(t), _ptr(c),
                             len(c), n_seeds, n_steps, minimum_length, _ptr(rows), _ptr(cols), _ptr(w))
        return rows, cols, w

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
    points = np.asarray(points, dtype=np.float32)
    points = points.reshape(-1, points.shape[-1] if points.ndim > 1 else 3)
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
    code = {"sin": 0, "cos": 1, "exp": 2, "log": 3, "exps2_cos": 4, "exps2_sinc": 5, "softplus": 6,
            "softplus_slope": 7, "softplus_inv_floor": 8, "cos2pi_u24": 9, "log_pos": 10, "exp_upto30": 11,
            "rsqrt_pos": 12}[which]
    lib().tgo_math(code, _ptr(x), x.size, _ptr(out))
    return out


# ---------------------------------------------------------------- boundary BVH

class BoundaryBvh:
    """A triangle surface and its BVH in the reference's array layout.

    ``build`` restates BaseDomain._set_boundary_data (domain.py:44-116):
    degenerate (zero or non-finite area) triangles are dropped, triangle
    bounds and centroids are float64, each node splits its triangles at the
    median of the centroids along the longest axis of its bounds (first axis
    on ties) after sorting them by that centroid coordinate, leaves hold at
    most 4 triangles, nodes are numbered in preorder and bounds are stored as
    float32.  The sort here is stable; NumPy's default argsort in the
    reference is not, so the two orders agree whenever no two centroids of a
    node are equal along its split axis.
    """

    LEAF_SIZE = 4

    def __init__(self, vertices4, triangles4, bounds_min, bounds_max, nodes, ordered):
        self.vertices = np.ascontiguousarray(vertices4, np.float32)
        self.triangles = np.ascontiguousarray(triangles4, np.uint32)
        self.bounds_min = np.ascontiguousarray(bounds_min, np.float32)
        self.bounds_max = np.ascontiguousarray(bounds_max, np.float32)
        self.nodes = np.ascontiguousarray(nodes, np.int32)
        self.ordered = np.ascontiguousarray(ordered, np.uint32)
        self.struct = Bvh(self.vertices.ctypes.data, self.triangles.ctypes.data, self.bounds_min.ctypes.data,
                          self.bounds_max.ctypes.data, self.nodes.ctypes.data, self.ordered.ctypes.data,
                          len(self.nodes))

    @classmethod
    def build(cls, vertices, faces):
        vertices = np.asarray(vertices, dtype=np.float64)
        faces = np.asarray(faces, dtype=np.uint32)
        tv = vertices[faces]
        area = 0.5 * np.linalg.norm(np.cross(tv[:, 1] - tv[:, 0], tv[:, 2] - tv[:, 0]), axis=1)
        faces = faces[np.isfinite(area) & (area > 0)]
        tv = vertices[faces]
        tmin, tmax = tv.min(axis=1), tv.max(axis=1)
        centroid = (tmin + tmax) * 0.5
        node_lo, node_hi, node_data, ordered = [], [], [], []

        def split(ids):
            me = len(node_data)
            node_lo.append(None)
            node_hi.append(None)
            node_data.append(None)
            lo, hi = tmin[ids].min(axis=0), tmax[ids].max(axis=0)
            if len(ids) <= cls.LEAF_SIZE:
                node_data[me] = (-1, -1, len(ordered), len(ids))
                ordered.extend(int(i) for i in ids)
            else:
                axis = int(np.argmax(hi - lo))
                ids = ids[np.argsort(centroid[ids, axis], kind="stable")]
                half = len(ids) // 2
                left = split(ids[:half])
                right = split(ids[half:])
                node_data[me] = (left, right, 0, 0)
            node_lo[me], node_hi[me] = lo, hi
            return me

        split(np.arange(len(faces), dtype=np.int64))
        v4 = np.ones((len(vertices), 4), np.float32)
        v4[:, :3] = vertices
        t4 = np.zeros((len(faces), 4), np.uint32)
        t4[:, :3] = faces
        bmin = np.zeros((len(node_lo), 4), np.float32)
        bmax = np.zeros((len(node_hi), 4), np.float32)
        bmin[:, :3] = np.asarray(node_lo)
        bmax[:, :3] = np.asarray(node_hi)
        return cls(v4, t4, bmin, bmax, np.asarray(node_data, np.int32), np.asarray(ordered, np.uint32))

    def segment_hits(self, starts, ends, n_threads=1):
        """bvh.cl:83-131 per row: (found, triangle, (n, 4) barycentric xyz + t)."""
        s4, e4 = _points4(starts), _points4(ends)
        n = len(s4)
        found = np.zeros(n, np.uint8)
        tri = np.zeros(n, np.uint32)
        hit = np.zeros((n, 4), np.float32)
        lib().tgo_segment_hits(ctypes.byref(self.struct), _ptr(s4), _ptr(e4), n, _ptr(found), _ptr(tri), _ptr(hit),
                               n_threads)
        return found.astype(bool), tri, hit

    def contains(self, points):
        pts = np.asarray(points, np.float32).reshape(-1, 3)
        f = lib().tgo_mesh_contains
        return np.array([f(ctypes.byref(self.struct), *map(float, q)) for q in pts], dtype=bool)


def boundary_seeds(vertices4, triangles4, cumulative, rng_seed, n):
    """domain.seed (domain.py:494-575): (n, 8) seeds on a boundary surface."""
    v = np.ascontiguousarray(vertices4, dtype=np.float32)
    t = np.ascontiguousarray(triangles4, dtype=np.uint32)
    c = np.ascontiguousarray(cumulative, dtype=np.float32)
    out = np.zeros((n, 8), np.float32)
    lib().tgo_boundary_seeds(_ptr(v), _ptr(t), _ptr(c), len(c), rng_seed & 0xFFFFFFFF, n, _ptr(out))
    return out
