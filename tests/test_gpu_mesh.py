"""Closed-surface (mesh) domain on the GPU vs the reference's hits and the oracle.

* segment hits through the C ABI equal the reference's bvh_segment_hit
  (tests/golden/bvh_reference.npz) bit for bit: found flag, triangle,
  barycentric coordinates and t;
* on the config-2 surface shape, segment hits, the tracking kernels'
  surface test (distance grid, per-cell leaf lists, walk) and the inside
  test equal the oracle's bit for bit;
* tracking with a mesh domain (dense one-thread-per-seed and packed
  persistent forms) equals the oracle's tracking loop bit for bit; the
  oracle walks the BVH for every step while the kernels skip the walk in
  empty distance-grid cells, so these tests also check that the skip never
  changes a result.
"""

from pathlib import Path

import numpy as np
import pytest

import tractography_b200 as tg
from oracle import oracle as O
from tractography_b200 import synthetic

from helpers import bits_equal, oracle_case

pytestmark = pytest.mark.gpu

G = np.load(Path(__file__).resolve().parent / "golden" / "bvh_reference.npz")


@pytest.mark.parametrize("name", ["soup", "sphere", "voxels"])
def test_segment_hits_match_reference(runtime, name):
    mesh = tg.domain.Mesh(G[f"{name}_input_vertices"], G[f"{name}_input_faces"])
    found, tri, hit = mesh.segment_hits(G[f"{name}_starts"], G[f"{name}_ends"], runtime)
    assert np.array_equal(found, G[f"{name}_found"])
    assert np.array_equal(tri, G[f"{name}_triangle"])
    assert bits_equal(hit, G[f"{name}_hit"])


def _surface(frequency=40, shape=(96, 96, 60)):
    v, f = synthetic.config2_surface(shape=shape, frequency=frequency)
    return v, f


def test_segment_hits_match_oracle_on_config2_surface(runtime):
    v, f = _surface()
    mesh = tg.domain.Mesh(v, f)
    bvh = O.BoundaryBvh.build(v, f)
    rng = np.random.default_rng(7)
    lo, hi = v.min(axis=0), v.max(axis=0)
    n = 20000
    k = rng.integers(0, len(f), n)
    p = v[f[k]].mean(axis=1) + rng.normal(0, 0.5, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    starts = np.concatenate([p, rng.uniform(lo - 5, hi + 5, (4000, 3))])
    ends = np.concatenate([p + d * rng.uniform(0, 0.6, (n, 1)), rng.uniform(lo - 5, hi + 5, (4000, 3))])
    got = mesh.segment_hits(starts, ends, runtime)
    want = bvh.segment_hits(starts, ends, n_threads=8)
    assert np.array_equal(got[0], want[0])
    assert np.array_equal(got[1], want[1])
    assert bits_equal(got[2], want[2])
    assert 0.1 < got[0].mean() < 0.9


@pytest.mark.parametrize("frequency", [40, 158])
def test_segments_blocked_match_oracle(runtime, frequency):
    """The tracking kernels' surface test (distance grid, per-cell leaf
    lists, walk) equals the found flag of the oracle's bvh_segment_hit walk
    on short segments near the surface (the leaf-list route), longer ones
    (the walk), far ones (the distance grid), segments from vertices and
    axis-parallel ones."""
    v, f = _surface(frequency=frequency)
    mesh = tg.domain.Mesh(v, f)
    bvh = O.BoundaryBvh.build(v, f)
    cell = 192.0 / (min(256, int(np.ceil(0.5 * np.sqrt(len(f))))) - 4)    # about the grid's cell
    rng = np.random.default_rng(frequency)
    lo, hi = v.min(axis=0), v.max(axis=0)
    n = 60000
    k = rng.integers(0, len(f), n)
    p = v[f[k]].mean(axis=1) + rng.normal(0, 0.4 * cell, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    length = np.concatenate([rng.uniform(0, 0.45 * cell, n - 10000), rng.uniform(0.5 * cell, 3 * cell, 10000)])
    starts = np.concatenate([p, v[f[k[:2000], 0]], rng.uniform(lo - 5, hi + 5, (3000, 3))]).astype(np.float32)
    ends = np.concatenate([p + d * length[:, None], v[f[k[:2000], 0]] + d[:2000] * 0.05,
                           rng.uniform(lo - 5, hi + 5, (3000, 3))]).astype(np.float32)
    ends[:3000, 1:] = starts[:3000, 1:]                            # parallel to the x axis
    got = mesh.segments_blocked(starts, ends, runtime)
    want = bvh.segment_hits(starts, ends, n_threads=8)[0].astype(bool)
    assert np.array_equal(got, want), np.flatnonzero(got != want)[:10]
    assert 0.05 < want.mean() < 0.6


def test_contains_matches_oracle(runtime):
    v, f = _surface()
    mesh = tg.domain.Mesh(v, f)
    bvh = O.BoundaryBvh.build(v, f)
    rng = np.random.default_rng(8)
    lo, hi = v.min(axis=0), v.max(axis=0)
    k = rng.integers(0, len(f), 3000)
    near = v[f[k]].mean(axis=1) + rng.normal(0, 0.05, (3000, 3))
    pts = np.concatenate([rng.uniform(lo - 3, hi + 3, (12000, 3)), near, v[:200]])
    got = tg.domain.contains(mesh, pts, runtime)
    want = bvh.contains(pts)
    assert np.array_equal(got, want)
    assert 0.2 < got.mean() < 0.8


def _dti_case(shape=(24, 24, 16), frequency=24, n_seeds=300):
    fod = synthetic.dti_field(shape=shape, seed=4)
    v, f = synthetic.config2_surface(shape=shape, frequency=frequency)
    mesh = tg.domain.Mesh(v, f)
    seeds = synthetic.seeds_inside(O.BoundaryBvh.build(v, f).contains, v.min(axis=0), v.max(axis=0), n_seeds,
                                   seed=3, chunk=4 * n_seeds)
    seeds[:3, 0] = -5.0                                     # three seeds outside the surface
    return tg.field.Image(fod), mesh, seeds


@pytest.mark.parametrize("kind", ["transport", "diffusion"])
def test_mesh_tracking_bit_exact(runtime, kind):
    field, mesh, seeds = _dti_case()
    model = tg.local.DiffusionTensorImaging()
    if kind == "transport":
        make = lambda: tg.algorithm.Transport(model, step_size=0.2, gamma=1.0)  # noqa: E731
    else:
        make = lambda: tg.algorithm.Diffusion(model, step_size=0.2, gamma=1.0, noise_variance=0.1,  # noqa: E731
                                              seed=21)
    n_steps = 160
    alg = make()
    dense, lengths = tg.tracking.tractogram_dense(alg, mesh, field, seeds, save_at=0.25,
                                                  maximum_streamline_length=n_steps * 0.25, runtime=runtime,
                                                  rng_seed=77)
    want, want_len = oracle_case(alg, mesh, field, rng_seed=77, save_at=0.25, n_steps=n_steps).tractogram(
        seeds, n_threads=8)
    assert np.array_equal(lengths, want_len)
    for i in range(len(seeds)):
        assert bits_equal(dense[i, : lengths[i]], want[i, : want_len[i]]), i
    assert np.all(lengths[:3] == 1) and lengths.max() > 20 and np.mean(lengths < n_steps) > 0.1

    alg2, twin = make(), make()
    result = tg.tracking.tractogram(alg2, mesh, field, seeds, save_at=0.25,
                                    maximum_streamline_length=n_steps * 0.25, runtime=runtime)
    want2, want_len2 = oracle_case(alg2, mesh, field, rng_seed=twin.get_rng_seed(), save_at=0.25,
                                   n_steps=n_steps).tractogram(seeds, n_threads=8)
    for i, s in enumerate(result.streamlines):
        assert bits_equal(s, want2[i, : want_len2[i], :3]), i


def test_tg_tractogram_with_mesh_domain(runtime):
    field, mesh, seeds = _dti_case(n_seeds=200)
    fod_img = tg.Nifti1Image(field.values, np.linalg.inv(field.inverse_affine))
    alg = tg.algorithm.Transport(tg.local.DiffusionTensorImaging(), step_size=0.2)
    got = tg.tractogram(fod_img, seeds, mesh, alg, save_at=0.25, maximum_streamline_length=20.0, batch_size=64,
                        runtime=runtime)
    want, want_len = oracle_case(alg, mesh, field, save_at=0.25, n_steps=80).tractogram(seeds)
    kept = [i for i in range(len(seeds)) if want_len[i] > 0]
    assert len(got.streamlines) == len(kept)
    for s, i in zip(got.streamlines, kept):
        assert bits_equal(s, want[i, : want_len[i], :3]), i
    info = mesh.info(runtime)
    assert info["triangles"] == len(mesh.faces) and info["nodes"] > 0 and min(info["grid"]) >= 5


@pytest.mark.parametrize("kind", ["image", "mesh"])
def test_boundary_seeds_bit_exact(runtime, kind):
    """domain.seed on the GPU equals the oracle (pinned to the reference's sampler)."""
    if kind == "image":
        fod, mask = synthetic.config0(n=16)
        dom = tg.domain.Image(mask)
    else:
        v, f = synthetic.config2_surface(shape=(24, 24, 16), frequency=20)
        dom = tg.domain.Mesh(v, f)
    for rng_seed in (0, 7, 0xFFFFFFFF):
        got = tg.domain.seed(dom, 20000, rng_seed=rng_seed, runtime=runtime)
        want = O.boundary_seeds(*dom.boundary_arrays(), rng_seed, 20000)
        assert bits_equal(got, want)


def test_tractogram_with_integer_seeds(runtime):
    fod, mask = synthetic.config0(n=16)
    alg = tg.algorithm.Transport(tg.local.RealSymmetricSphericalHarmonics(45), step_size=0.2)
    t = tg.tractogram(fod, 300, mask, alg, save_at=0.25, maximum_streamline_length=20.0, runtime=runtime)
    assert len(t.streamlines) == 300
    starts = np.array([s[0] for s in t.streamlines])
    assert np.all(tg.domain.Image(mask).contains(starts))
