#!/usr/bin/env python3
"""Golden vectors for the boundary BVH, from the reference itself.

Run where the reference sources are available (oracle.build_ref.reference_root)
after ``python oracle/build_ref.py``; writes tests/golden/bvh_reference.npz.

Three triangle sets:

* ``soup``: 1500 separate random triangles (no shared vertices), so no two
  triangle centroids tie and the reference's BVH arrays are fully
  determined by its algorithm;
* ``sphere``: a geodesic sphere (frequency 8, 1280 triangles) with seeded
  vertex jitter;
* ``voxels``: the voxel-face boundary the reference builds for an image
  domain (domain.py:219-264) of a seeded blob mask under an affine with a
  reflection.

Closed meshes have tied centroids by construction (neighbouring faces share
their extreme vertices along an axis).  The reference sorts with NumPy's
default argsort, which is not stable (introsort, or a SIMD sort on CPUs
with AVX-512), so on those meshes its tree depends on the machine; they pin
traversal results, the soup pins the tree.

For each: the reference's BVH arrays and normalised cumulative triangle
areas (BaseDomain._set_boundary_data,
domain.py:44-116, run on the reference's own Python code), and for a set of
seeded segments (near-surface steps, long chords, axis-parallel and
zero-length segments) the output of the reference's bvh_segment_hit
(utils/bvh.cl:83-131) compiled on the CPU (oracle/_ref).
"""

from __future__ import annotations

import argparse
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from oracle.build_ref import reference_root  # noqa: E402
from oracle.refstubs import install_stubs  # noqa: E402


def segments(rng, vertices, faces, scale):
    tri = vertices[faces]
    n_near, n_chord, n_axis = 1500, 500, 200
    k = rng.integers(0, len(faces), n_near)
    r1, r2 = np.sqrt(rng.uniform(size=n_near)), rng.uniform(size=n_near)
    p = (1 - r1)[:, None] * tri[k, 0] + (r1 * (1 - r2))[:, None] * tri[k, 1] + (r1 * r2)[:, None] * tri[k, 2]
    normal = np.cross(tri[k, 1] - tri[k, 0], tri[k, 2] - tri[k, 0])
    normal /= np.linalg.norm(normal, axis=1, keepdims=True)
    start = p + normal * rng.uniform(-0.3, 0.3, (n_near, 1)) * scale
    d = rng.normal(size=(n_near, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    end = start + d * rng.uniform(0.0, 0.5, (n_near, 1)) * scale
    lo, hi = vertices.min(axis=0), vertices.max(axis=0)
    pad = 0.2 * (hi - lo)
    c0 = rng.uniform(lo - pad, hi + pad, (n_chord, 3))
    c1 = rng.uniform(lo - pad, hi + pad, (n_chord, 3))
    a0 = rng.uniform(lo, hi, (n_axis, 3))
    a1 = a0.copy()
    axis = rng.integers(0, 3, n_axis)
    a1[np.arange(n_axis), axis] = rng.uniform(lo[axis] - pad[axis], hi[axis] + pad[axis])
    z = rng.uniform(lo, hi, (20, 3))
    starts = np.concatenate([start, c0, a0, z]).astype(np.float32)
    ends = np.concatenate([end, c1, a1, z]).astype(np.float32)
    return starts, ends


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=str(reference_root()))
    args = ap.parse_args()
    install_stubs(Path(args.reference))
    import tractography as ref  # noqa: E402  (the reference package)

    from oracle import reference as R
    from tractography_b200 import synthetic

    if not R.available():
        raise SystemExit("build oracle/_ref first: python oracle/build_ref.py")
    rng = np.random.default_rng(20261204)
    Trimesh = sys.modules["trimesh"].Trimesh
    out = {}

    n_soup = 1500
    centre = rng.uniform([0, 0, 0], [60, 50, 40], (n_soup, 1, 3))
    sv = (centre + rng.normal(0.0, 1.5, (n_soup, 3, 3))).reshape(-1, 3)
    sf = np.arange(3 * n_soup, dtype=np.uint32).reshape(-1, 3)
    soup = types.SimpleNamespace()
    ref.domain.BaseDomain._set_boundary_data(soup, Trimesh(sv, sf))
    out["soup_input_vertices"], out["soup_input_faces"] = sv, sf

    v, f = synthetic.geodesic_sphere(8)
    v = v * np.array([30.0, 24.0, 18.0]) + rng.normal(0.0, 0.05, v.shape) + np.array([40.0, 35.0, 25.0])
    sphere = types.SimpleNamespace()
    ref.domain.BaseDomain._set_boundary_data(sphere, Trimesh(v, f))
    out["sphere_input_vertices"], out["sphere_input_faces"] = v, f.astype(np.uint32)
    holders = {"soup": (soup, sv, sf, 2.0), "sphere": (sphere, v, f, 2.0)}

    mask = np.zeros((7, 6, 5), bool)
    mask[1:6, 1:5, 1:4] = rng.uniform(size=(5, 4, 3)) < 0.7
    mask[3, 2, 2] = True
    affine = np.array([[-1.5, 0.1, 0.0, 10.0], [0.0, 1.25, 0.2, -4.0], [0.05, 0.0, 2.0, 3.0], [0, 0, 0, 1]])
    img = sys.modules["nibabel.nifti1"].Nifti1Image(mask.astype(np.uint8), affine)
    voxels = ref.domain.Image(img)
    out["voxels_mask"], out["voxels_affine"] = mask, affine
    bv, bf = np.asarray(voxels.boundary.vertices), np.asarray(voxels.boundary.faces)
    out["voxels_input_vertices"], out["voxels_input_faces"] = bv, bf.astype(np.uint32)
    holders["voxels"] = (voxels, bv, bf, 1.0)

    for name, (h, vv, ff, scale) in holders.items():
        arrays = {
            "vertices": h.boundary_vertices, "triangles": h.boundary_indices,
            "bounds_min": h.boundary_bvh_bounds_min, "bounds_max": h.boundary_bvh_bounds_max,
            "nodes": h.boundary_bvh_nodes, "ordered_triangles": h.boundary_bvh_triangles,
        }
        for key, a in arrays.items():
            out[f"{name}_{key}"] = np.asarray(a)
        out[f"{name}_cumulative"] = np.asarray(h.boundary_cumulative_areas)
        s, e = segments(rng, vv, ff, scale)
        found, tri, hit = R.bvh_hits(*arrays.values(), s, e)
        out[f"{name}_starts"], out[f"{name}_ends"] = s, e
        out[f"{name}_found"], out[f"{name}_triangle"], out[f"{name}_hit"] = found, tri, hit
        print(f"{name}: {len(ff)} faces, {len(arrays['nodes'])} nodes, {found.sum()} of {len(s)} segments hit")
    np.savez_compressed(HERE / "bvh_reference.npz", **out)
    print("wrote", HERE / "bvh_reference.npz")


if __name__ == "__main__":
    main()
