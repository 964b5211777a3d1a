"""Tracking domains (reference ``tractography/domain.py``).

``Image`` is the nonzero-voxel domain: a point is inside when its nearest
voxel, ``floor(A^-1 p + 0.5)`` (half-open cells ``[i - 0.5, i + 0.5)``), is
inside the image and nonzero (domain.py:358-382).  On the GPU the mask is a
``tg_domain`` of uint8 created once per runtime.

The reference also builds a voxel-face boundary mesh and a BVH in every
``Image`` constructor for boundary seeding and connectome end points
(domain.py:44-116, 219-264); the streamline tracker never reads them, so
``Image`` builds its boundary only when ``seed`` needs it.

``Mesh`` makes a closed triangle surface the domain.  Its BVH is the
reference's boundary BVH (median split of domain.py:72-116, traversal of
utils/bvh.cl:83-131), built natively on the host and kept on the device: a
seed is inside by a three-ray crossing-parity vote, and a streamline stops
at the first step whose segment from the previous point hits the surface.
"""

from __future__ import annotations

import ctypes
from abc import ABC, abstractmethod

import numpy as np

from . import _lib
from .nifti import apply_affine


class BaseDomain(ABC):
    """Region in which tracking continues (domain.py:20-216)."""

    @abstractmethod
    def contains(self, points) -> np.ndarray:
        """Authoritative membership test for (n, 3) world-space points."""

    def boundary_mesh(self):
        """(vertices (V, 3) float64, faces (F, 3)) of the domain's boundary surface."""
        raise NotImplementedError(f"{type(self).__name__} has no boundary surface")

    @property
    def boundary(self):
        """The boundary surface (``vertices``, ``faces``), as the reference's
        ``domain.boundary`` mesh; rows and columns of the boundary connectome
        follow its vertex order."""
        from types import SimpleNamespace

        vertices, faces = self.boundary_mesh()
        return SimpleNamespace(vertices=vertices, faces=faces)

    def boundary_bvh(self):
        """The boundary surface as a ``Mesh`` (its BVH answers end-segment hits)."""
        cached = getattr(self, "_boundary_bvh", None)
        if cached is None:
            if isinstance(self, Mesh):
                cached = self
            else:
                vertices, faces = self.boundary_mesh()
                cached = Mesh(vertices, faces)
            self._boundary_bvh = cached
        return cached

    def boundary_arrays(self):
        """The boundary sampler's arrays (domain.py:44-70): float32 vertices
        (V, 4), uint32 kept faces (T, 4) and float32 normalised cumulative
        areas (T,), faces of zero or non-finite area dropped."""
        cached = getattr(self, "_boundary_arrays", None)
        if cached is not None:
            return cached
        vertices, faces = self.boundary_mesh()
        vertices = np.asarray(vertices, dtype=np.float64)
        faces = np.asarray(faces, dtype=np.uint32)
        if len(faces) == 0:
            raise ValueError("The boundary mesh must contain at least one triangle.")
        t = vertices[faces]
        area = 0.5 * np.linalg.norm(np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0]), axis=1)
        valid = np.isfinite(area) & (area > 0)
        faces, area = faces[valid], area[valid]
        if len(faces) == 0:
            raise ValueError("The boundary mesh must contain a non-degenerate triangle.")
        v4 = np.ones((len(vertices), 4), np.float32)
        v4[:, :3] = vertices
        f4 = np.zeros((len(faces), 4), np.uint32)
        f4[:, :3] = faces
        total = float(np.sum(area, dtype=np.float64))
        if not np.isfinite(total) or total <= 0:
            raise ValueError("The boundary mesh must have a finite, positive area.")
        cumulative = np.cumsum(area / total).astype(np.float32)
        cumulative[-1] = 1.0
        self._boundary_arrays = (v4, f4, cumulative)
        return self._boundary_arrays


def voxel_boundary_mesh(mask, affine):
    """Surface of the union of the occupied voxel cells (domain.py:219-264).

    Voxel centres have integer coordinates and each voxel occupies a unit
    cell; a square face (two triangles) is emitted where an occupied voxel
    meets an empty one or the outside of the array, wound outward (reversed
    when the affine reflects).  Vertices are the distinct cell corners in
    lexicographic order of their voxel coordinates."""
    mask = np.asarray(mask, dtype=bool)
    # (direction, corner offsets in doubled voxel units), outward winding
    sides = (
        ((-1, 0, 0), ((-1, -1, -1), (-1, -1, 1), (-1, 1, 1), (-1, 1, -1))),
        ((1, 0, 0), ((1, -1, -1), (1, 1, -1), (1, 1, 1), (1, -1, 1))),
        ((0, -1, 0), ((-1, -1, -1), (1, -1, -1), (1, -1, 1), (-1, -1, 1))),
        ((0, 1, 0), ((-1, 1, -1), (-1, 1, 1), (1, 1, 1), (1, 1, -1))),
        ((0, 0, -1), ((-1, -1, -1), (-1, 1, -1), (1, 1, -1), (1, -1, -1))),
        ((0, 0, 1), ((-1, -1, 1), (1, -1, 1), (1, 1, 1), (-1, 1, 1))),
    )
    padded = np.pad(mask, 1, mode="constant", constant_values=False)
    quads = []
    for step, corners in sides:
        neighbour = padded[tuple(slice(1 + d, 1 + d + n) for d, n in zip(step, mask.shape))]
        exposed = np.argwhere(mask & ~neighbour)
        if len(exposed):
            quads.append(2 * exposed[:, None, :] + np.asarray(corners, dtype=np.int64))
    doubled = np.concatenate(quads, axis=0).reshape(-1, 3)
    corners, index = np.unique(doubled, axis=0, return_inverse=True)
    q = index.reshape(-1, 4)
    faces = np.concatenate((q[:, (0, 1, 2)], q[:, (0, 2, 3)]), axis=0)
    affine = np.asarray(affine, dtype=np.float64)
    vertices = apply_affine(affine, corners.astype(np.float64) * 0.5)
    if np.linalg.det(affine[:3, :3]) < 0:
        faces = faces[:, [0, 2, 1]]
    return vertices, faces


class Image(BaseDomain):
    """Domain of the nonzero voxels of a 3D image (domain.py:267-430)."""

    def __init__(self, image_data):
        if image_data.ndim != 3:
            raise ValueError("Only 3D images are supported for image domains.")
        self.values = np.ascontiguousarray(image_data.get_fdata() != 0, dtype=np.int32)
        self.dims = np.ascontiguousarray((*image_data.shape, 0), dtype=np.uint32)
        affine = image_data.affine
        self.affine = np.asarray(affine if affine is not None else np.eye(4), dtype=np.float64)
        self.inverse_affine = np.ascontiguousarray(np.linalg.inv(self.affine), dtype=np.float32)
        if not np.any(self.values):
            raise ValueError("Image domain must contain at least one nonzero voxel.")
        self._device = {}

    def boundary_mesh(self):
        """The voxel-face surface of the mask (domain.py:219-264), built on first use."""
        cached = getattr(self, "_boundary_mesh", None)
        if cached is None:
            cached = voxel_boundary_mesh(self.values != 0, self.affine)
            self._boundary_mesh = cached
        return cached

    def contains(self, points) -> np.ndarray:
        """NumPy reference of domain.py:400-430."""
        voxel = np.floor(apply_affine(self.inverse_affine, points) + 0.5).astype(int)
        x, y, z = voxel[:, :3].T
        width, height, depth = self.values.shape
        inside = (0 <= x) & (x < width) & (0 <= y) & (y < height) & (0 <= z) & (z < depth)
        result = np.zeros(x.shape, dtype=np.bool_)
        result[inside] = self.values[x[inside], y[inside], z[inside]] != 0
        return result

    def device(self, runtime):
        """The ``tg_domain`` of this mask for ``runtime``."""
        key = id(runtime)
        obj = self._device.get(key)
        if obj is None:
            from .runtime import DeviceObject

            mask = np.ascontiguousarray(self.values != 0, dtype=np.uint8)
            nx, ny, nz = (int(v) for v in mask.shape)
            handle = ctypes.c_void_p()
            with runtime.device_scope():
                _lib.check(runtime.lib.tg_domain_create(
                    mask.ctypes.data_as(ctypes.c_void_p), nx, ny, nz,
                    self.inverse_affine.ctypes.data_as(ctypes.c_void_p),
                    ctypes.c_void_p(runtime.stream_handle), ctypes.byref(handle)))
            obj = DeviceObject(handle, runtime.lib.tg_domain_destroy)
            self._device[key] = obj
        return obj.handle


class Mesh(BaseDomain):
    """Domain bounded by a closed, outward-wound triangle surface.

    ``Mesh(vertices, faces)`` with (V, 3) vertices and (F, 3) vertex indices,
    or ``Mesh(mesh)`` for any object with ``vertices`` and ``faces`` (a
    trimesh.Trimesh, for example).  Faces of zero or non-finite area are
    dropped as in domain.py:49-57.
    """

    def __init__(self, vertices, faces=None):
        if faces is None:
            vertices, faces = vertices.vertices, vertices.faces
        self.vertices = np.ascontiguousarray(vertices, dtype=np.float64)
        self.faces = np.ascontiguousarray(faces, dtype=np.uint32)
        if self.vertices.ndim != 2 or self.vertices.shape[1] != 3:
            raise ValueError("vertices must have shape (n_vertices, 3)")
        if self.faces.ndim != 2 or self.faces.shape[1] != 3:
            raise ValueError("faces must have shape (n_faces, 3)")
        if len(self.faces) == 0:
            raise ValueError("The boundary mesh must contain at least one triangle.")
        if self.faces.max() >= len(self.vertices):
            raise ValueError("face vertex index out of range")
        self._device = {}

    def boundary_mesh(self):
        return self.vertices, self.faces

    def bvh_arrays(self) -> dict:
        """The boundary BVH in the reference's layout (domain.py:100-116).

        Built by the library on the host: ``vertices`` (V, 4) float32,
        ``triangles`` (T, 4) uint32 of the kept faces, ``bounds_min`` and
        ``bounds_max`` (N, 4) float32, ``nodes`` (N, 4) int32 (left, right,
        first, count) and ``ordered_triangles`` (T,) uint32.
        """
        lib = _lib.load()
        nt, nn = ctypes.c_uint32(), ctypes.c_uint32()
        P = ctypes.c_void_p
        v, f = self.vertices, self.faces
        args = (v.ctypes.data_as(P), len(v), f.ctypes.data_as(P), len(f), ctypes.byref(nt), ctypes.byref(nn))
        _lib.check(lib.tg_bvh_build_host(*args, None, None, None, None, None, None))
        out = {
            "vertices": np.empty((len(v), 4), np.float32),
            "triangles": np.empty((nt.value, 4), np.uint32),
            "bounds_min": np.empty((nn.value, 4), np.float32),
            "bounds_max": np.empty((nn.value, 4), np.float32),
            "nodes": np.empty((nn.value, 4), np.int32),
            "ordered_triangles": np.empty(nt.value, np.uint32),
        }
        _lib.check(lib.tg_bvh_build_host(*args, *(a.ctypes.data_as(P) for a in out.values())))
        return out

    def contains(self, points) -> np.ndarray:
        """Inside test on the GPU (three-ray crossing-parity vote)."""
        return contains(self, points)

    def device(self, runtime):
        """The ``tg_domain`` of this surface for ``runtime``."""
        key = id(runtime)
        obj = self._device.get(key)
        if obj is None:
            from .runtime import DeviceObject

            handle = ctypes.c_void_p()
            with runtime.device_scope():
                _lib.check(runtime.lib.tg_domain_create_mesh(
                    self.vertices.ctypes.data_as(ctypes.c_void_p), len(self.vertices),
                    self.faces.ctypes.data_as(ctypes.c_void_p), len(self.faces),
                    ctypes.c_void_p(runtime.stream_handle), ctypes.byref(handle)))
            obj = DeviceObject(handle, runtime.lib.tg_domain_destroy)
            self._device[key] = obj
        return obj.handle

    def info(self, runtime=None) -> dict:
        """Triangles, BVH nodes, distance-grid cells and device bytes."""
        from .runtime import default_runtime

        runtime = runtime or default_runtime()
        nt, nn, nbytes = ctypes.c_uint32(), ctypes.c_uint32(), ctypes.c_uint64()
        grid = (ctypes.c_uint32 * 3)()
        _lib.check(runtime.lib.tg_mesh_info(self.device(runtime), ctypes.byref(nt), ctypes.byref(nn), grid,
                                            ctypes.byref(nbytes)))
        return {"triangles": nt.value, "nodes": nn.value, "grid": tuple(grid), "device_bytes": nbytes.value}

    def segment_hits(self, starts, ends, runtime=None):
        """bvh_segment_hit (utils/bvh.cl:83-131) per segment on the GPU.

        Returns (found, triangle index among the kept faces, (n, 4)
        barycentric coordinates and segment parameter t)."""
        from .runtime import default_runtime

        import torch

        runtime = runtime or default_runtime()
        n = len(starts)
        s4 = np.zeros((n, 4), np.float32)
        e4 = np.zeros((n, 4), np.float32)
        s4[:, :3], e4[:, :3] = np.asarray(starts)[:, :3], np.asarray(ends)[:, :3]
        if n == 0:
            return np.zeros(0, bool), np.zeros(0, np.uint32), np.zeros((0, 4), np.float32)
        with runtime.device_scope():
            handle = self.device(runtime)
            ds, de = runtime.to_device(s4), runtime.to_device(e4)
            found = runtime.empty((n,), torch.uint8)
            tri = runtime.empty((n,), torch.int32)
            hit = runtime.empty((n, 4), torch.float32)
            _lib.check(runtime.lib.tg_mesh_segment_hits(
                handle, ctypes.c_void_p(ds.data_ptr()), ctypes.c_void_p(de.data_ptr()), n,
                ctypes.c_void_p(found.data_ptr()), ctypes.c_void_p(tri.data_ptr()), ctypes.c_void_p(hit.data_ptr()),
                ctypes.c_void_p(runtime.stream_handle)))
            return (found.cpu().numpy().astype(bool), tri.cpu().numpy().view(np.uint32),
                    hit.cpu().numpy())

    def segments_blocked(self, starts, ends, runtime=None) -> np.ndarray:
        """Whether each segment hits the surface, computed as the tracking
        kernels' domain test computes it (the found flag of
        bvh_segment_hit, utils/bvh.cl:83-131)."""
        from .runtime import default_runtime

        import torch

        runtime = runtime or default_runtime()
        n = len(starts)
        if n == 0:
            return np.zeros(0, bool)
        s4 = np.zeros((n, 4), np.float32)
        e4 = np.zeros((n, 4), np.float32)
        s4[:, :3], e4[:, :3] = np.asarray(starts)[:, :3], np.asarray(ends)[:, :3]
        with runtime.device_scope():
            handle = self.device(runtime)
            ds, de = runtime.to_device(s4), runtime.to_device(e4)
            out = runtime.empty((n,), torch.uint8)
            _lib.check(runtime.lib.tg_mesh_segments_blocked(
                handle, ctypes.c_void_p(ds.data_ptr()), ctypes.c_void_p(de.data_ptr()), n,
                ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(runtime.stream_handle)))
            return out.cpu().numpy().astype(bool)


def contains(domain: BaseDomain, points, runtime=None) -> np.ndarray:
    """GPU membership test (domain.py:433-491)."""
    points = np.asarray(points)
    n = points.shape[0]
    if n == 0:
        return np.array([], dtype=np.bool_)
    if not isinstance(domain, (Image, Mesh)):
        raise NotImplementedError(f"{type(domain).__name__} has no compiled CUDA code path")
    from .runtime import default_runtime

    runtime = runtime or default_runtime()
    import torch

    pts = np.zeros((n, 4), dtype=np.float32)
    pts[:, :3] = points
    pts[:, 3] = 1.0
    with runtime.device_scope():
        handle = domain.device(runtime)
        d_pts = runtime.to_device(pts)
        d_out = runtime.empty((n,), torch.uint8)
        _lib.check(runtime.lib.tg_domain_contains(handle, ctypes.c_void_p(d_pts.data_ptr()), n,
                                                  ctypes.c_void_p(d_out.data_ptr()),
                                                  ctypes.c_void_p(runtime.stream_handle)))
        return d_out.cpu().numpy().astype(bool)


def seed(domain: BaseDomain, n_seeds: int, rng_seed=None, runtime=None) -> np.ndarray:
    """Seeds uniform over the boundary surface area, pointing inward (domain.py:494-575).

    Seed i draws from the MWC64X stream rng_init(rng_seed, i): a uniform
    target selects the triangle through the normalised cumulative areas, two
    more give a uniform point in it; the orientation is the inward normal
    and the point sits 1e-4 along it.  Returns (n_seeds, 8) float32 rows."""
    if not isinstance(n_seeds, (int, np.integer)) or n_seeds < 0:
        raise ValueError("n_seeds must be a non-negative integer.")
    if n_seeds == 0:
        return np.empty((0, 8), dtype=np.float32)
    if rng_seed is None:
        rng_seed = int(np.random.default_rng().integers(0, 2**32, dtype=np.uint32))
    rng_seed = int(rng_seed) % 2**32
    v4, f4, cumulative = domain.boundary_arrays()
    from .runtime import default_runtime

    runtime = runtime or default_runtime()
    import torch

    with runtime.device_scope():
        dv, df, dc = runtime.to_device(v4), runtime.to_device(f4), runtime.to_device(cumulative)
        out = runtime.empty((int(n_seeds), 8), torch.float32)
        _lib.check(runtime.lib.tg_boundary_seeds(
            ctypes.c_void_p(dv.data_ptr()), len(v4), ctypes.c_void_p(df.data_ptr()),
            ctypes.c_void_p(dc.data_ptr()), len(f4), rng_seed, int(n_seeds), ctypes.c_void_p(out.data_ptr()),
            ctypes.c_void_p(runtime.stream_handle)))
        return out.cpu().numpy()
