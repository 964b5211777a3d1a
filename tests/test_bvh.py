"""Boundary BVH and the closed-surface domain on the CPU.

Pins, against tests/golden/bvh_reference.npz (made by make_bvh_golden.py
from the reference's own Python BVH build and its bvh.cl traversal compiled
on the CPU):

* the oracle's restated build and the library's native build reproduce the
  reference's BVH arrays bit for bit on a triangle soup, where no centroids
  tie and the reference's split order is determined, and agree with each
  other everywhere (both sort stably; the reference's NumPy argsort orders
  tied centroids in a machine-dependent way);
* the oracle's restated traversal reproduces the reference's hits (found,
  triangle, barycentric coordinates, t) bit for bit on the reference's
  trees, and the traversal of our stably sorted trees gives the same hits on
  the closed surfaces, whose centroids tie;
* the inside test and the mesh-domain tracking loop of the oracle behave as
  their definitions say on an analytic sphere.
"""

from pathlib import Path

import numpy as np
import pytest

import tractography_b200 as tg
from oracle import oracle as O
from tractography_b200 import synthetic

G = np.load(Path(__file__).resolve().parent / "golden" / "bvh_reference.npz")
KEYS = ("vertices", "triangles", "bounds_min", "bounds_max", "nodes", "ordered_triangles")


def _bits(a):
    a = np.ascontiguousarray(a)
    return a.view(np.uint32) if a.dtype == np.float32 else a


def _same(a, b):
    return a.shape == b.shape and np.array_equal(_bits(a), _bits(b))


def _ref_arrays(name):
    return {k: G[f"{name}_{k}"] for k in KEYS}


def _oracle_arrays(b):
    return dict(zip(KEYS, (b.vertices, b.triangles, b.bounds_min, b.bounds_max, b.nodes, b.ordered)))


def test_oracle_build_matches_reference_build():
    ref = _ref_arrays("soup")
    b = O.BoundaryBvh.build(G["soup_input_vertices"], G["soup_input_faces"])
    got = _oracle_arrays(b)
    for k in KEYS:
        assert _same(got[k], ref[k]), k


def test_native_build_matches_reference_build():
    ref = _ref_arrays("soup")
    got = tg.domain.Mesh(G["soup_input_vertices"], G["soup_input_faces"]).bvh_arrays()
    for k in KEYS:
        assert _same(got[k], ref[k]), k


@pytest.mark.parametrize("name", ["soup", "sphere", "voxels"])
def test_native_build_matches_oracle_build(name):
    v, f = G[f"{name}_input_vertices"], G[f"{name}_input_faces"]
    got = tg.domain.Mesh(v, f).bvh_arrays()
    want = _oracle_arrays(O.BoundaryBvh.build(v, f))
    for k in KEYS:
        assert _same(got[k], want[k]), k
    # the reference's vertex and kept-face arrays do not depend on the sort
    ref = _ref_arrays(name)
    assert _same(got["vertices"], ref["vertices"]) and _same(got["triangles"], ref["triangles"])


def test_native_build_drops_degenerate_faces_and_rejects_bad_input():
    v, f = synthetic.geodesic_sphere(2)
    v = np.concatenate([v, v[:1]])                           # duplicate of vertex 0
    f = np.concatenate([f, [[0, 1, len(v) - 1]], [[3, 3, 4]]]).astype(np.uint32)
    arrays = tg.domain.Mesh(v, f).bvh_arrays()
    assert len(arrays["triangles"]) == len(f) - 2
    with pytest.raises(ValueError):
        tg.domain.Mesh(v, np.array([[0, 1, len(v)]]))
    with pytest.raises(ValueError):
        tg.domain.Mesh(v, np.zeros((0, 3), np.uint32))
    flat = np.zeros((3, 3))
    with pytest.raises(ValueError, match="non-degenerate"):
        tg.domain.Mesh(flat, np.array([[0, 1, 2]])).bvh_arrays()


def _check_hits(got, name):
    found, tri, hit = got
    assert np.array_equal(found, G[f"{name}_found"])
    assert np.array_equal(tri, G[f"{name}_triangle"])
    assert _same(hit, G[f"{name}_hit"])
    assert 0.2 < found.mean() < 0.8


@pytest.mark.parametrize("name", ["soup", "sphere", "voxels"])
def test_oracle_traversal_matches_reference_hits(name):
    ref = _ref_arrays(name)
    b = O.BoundaryBvh(*(ref[k] for k in KEYS))
    _check_hits(b.segment_hits(G[f"{name}_starts"], G[f"{name}_ends"]), name)


@pytest.mark.parametrize("name", ["sphere", "voxels"])
def test_stable_tree_gives_the_reference_hits(name):
    b = O.BoundaryBvh.build(G[f"{name}_input_vertices"], G[f"{name}_input_faces"])
    _check_hits(b.segment_hits(G[f"{name}_starts"], G[f"{name}_ends"]), name)


def test_oracle_contains_on_a_sphere():
    v, f = synthetic.geodesic_sphere(16)
    b = O.BoundaryBvh.build(v * 10.0, f)
    rng = np.random.default_rng(3)
    p = rng.uniform(-11, 11, (4000, 3))
    r = np.linalg.norm(p, axis=1)
    clear = (r < 9.8) | (r > 10.05)                           # away from the faceted surface
    got = b.contains(p)
    assert np.array_equal(got[clear], r[clear] < 10.0)


def test_oracle_mesh_tracking_stops_at_the_surface():
    # uniform tensor field along x inside a sphere of radius 10 mm
    D = np.zeros((24, 24, 24, 6), np.float32)
    D[..., 0], D[..., 1], D[..., 2] = 1.7e-3, 0.3e-3, 0.3e-3
    affine = np.diag([1.0, 1.0, 1.0, 1.0])
    affine[:3, 3] = -11.5
    field = tg.field.Image(tg.Nifti1Image(D, affine))
    v, f = synthetic.geodesic_sphere(24)
    mesh = tg.domain.Mesh(v * 10.0, f)
    seeds = np.zeros((5, 8), np.float32)
    seeds[:, 0] = [-6.0, -2.0, 0.0, 3.0, 12.0]               # the last seed is outside
    seeds[:, 3] = 1.0
    seeds[:, 4] = 1.0
    alg = tg.algorithm.Transport(tg.local.DiffusionTensorImaging(), step_size=0.05, gamma=1.0)
    from helpers import oracle_case

    pts, n = oracle_case(alg, mesh, field, save_at=0.05, n_steps=2000).tractogram(seeds)
    assert n[-1] == 1
    # as in the reference loop (tracking.py:121-147), the point saved by the
    # step that leaves the domain is the last one: it lies just past the
    # (faceted, radius <= 10) surface, the point before it inside
    last = pts[np.arange(4), n[:4] - 1, 0]
    before = pts[np.arange(4), n[:4] - 2, 0]
    assert np.all(last > 9.95) and np.all(last <= 10.0 + 0.05)
    assert np.all(before <= 10.0) and np.all(last - before > 0.049)


def test_voxel_boundary_mesh_matches_reference():
    """domain.py:219-264 restated: same vertices (float64) and faces."""
    img = tg.Nifti1Image(G["voxels_mask"].astype(np.uint8), G["voxels_affine"])
    v, f = tg.domain.Image(img).boundary_mesh()
    assert np.array_equal(v, G["voxels_input_vertices"])
    assert np.array_equal(f, G["voxels_input_faces"])


@pytest.mark.parametrize("name", ["sphere", "voxels"])
def test_boundary_arrays_match_reference(name):
    """domain.py:44-70: kept faces, float32 vertices and cumulative areas bit for bit."""
    if name == "voxels":
        dom = tg.domain.Image(tg.Nifti1Image(G["voxels_mask"].astype(np.uint8), G["voxels_affine"]))
    else:
        dom = tg.domain.Mesh(G["sphere_input_vertices"], G["sphere_input_faces"])
    v4, f4, cum = dom.boundary_arrays()
    assert _same(v4, G[f"{name}_vertices"]) and _same(f4, G[f"{name}_triangles"])
    assert _same(cum, G[f"{name}_cumulative"])


def test_oracle_boundary_seeds_are_on_the_surface_pointing_inward():
    v, f = synthetic.geodesic_sphere(12)
    dom = tg.domain.Mesh(v * 10.0, f)
    s = O.boundary_seeds(*dom.boundary_arrays(), 99, 5000)
    r = np.linalg.norm(s[:, :3].astype(np.float64), axis=1)
    assert np.all(r < 10.0) and np.all(r > 9.9)               # on the faceted surface, 1e-4 inside
    assert np.all(np.einsum("ij,ij->i", s[:, 4:7], s[:, :3]) < 0)   # inward
    assert np.allclose(np.linalg.norm(s[:, 4:7], axis=1), 1.0, atol=1e-6)
    assert np.all(s[:, 3] == 1.0) and np.all(s[:, 7] == 0.0)
