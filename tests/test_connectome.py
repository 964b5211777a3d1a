"""Boundary connectome: host logic and the oracle on the reference tests' cases."""

import numpy as np
import pytest
from scipy.sparse import csr_matrix

import tractography_b200 as tg
from oracle import oracle as O
from tractography_b200.tracking import contributions_to_matrix

import data
from helpers import oracle_case


def _oracle_matrix(alg, domain, field, n_seeds, max_len, min_len=0.0, rng_seed=0):
    boundary = domain.boundary_bvh()
    bvh = O.BoundaryBvh.build(boundary.vertices, boundary.faces)
    n_steps = int(np.floor(max_len / alg.step_size))
    rows, cols, w = oracle_case(alg, domain, field, rng_seed=rng_seed).connectome(
        bvh, domain.boundary_arrays(), n_seeds, n_steps, min_len)
    return contributions_to_matrix(rows, cols, w, len(domain.boundary.vertices))


def test_connectome_zero_seeds_returns_empty_csr_without_gpu():
    """test/test_tracking.py:212-224."""
    domain = tg.domain.Image(tg.Nifti1Image(np.ones((1, 1, 1), np.uint8), np.eye(4)))
    field = tg.field.Image(tg.Nifti1Image(np.zeros((1, 1, 1, 15), np.float32), np.eye(4)))
    alg = tg.algorithm.Transport(tg.local.RealSymmetricSphericalHarmonics(15))
    m = tg.tracking.connectome(alg, domain, field, n_seeds=0)
    assert isinstance(m, csr_matrix) and m.shape == (len(domain.boundary.vertices),) * 2 and m.nnz == 0


def test_oracle_connectome_piecewise_linear_matrix():
    """test/test_tracking.py:183-209 on the oracle."""
    domain = tg.domain.Image(tg.Nifti1Image(np.ones((1, 1, 1), np.uint8), np.eye(4)))
    f = np.zeros((1, 1, 1, 15), np.float32)
    f[..., 0] = 1.0
    field = tg.field.Image(tg.Nifti1Image(f, np.eye(4)))
    alg = tg.algorithm.Transport(tg.local.RealSymmetricSphericalHarmonics(15), step_size=0.1, gamma=0.0)
    m = _oracle_matrix(alg, domain, field, 16, 2.0)
    assert m.shape == (8, 8) and m.nnz > 0 and m.dtype == np.float32
    assert 0.0 < m.sum() <= 16.0 + 1e-5


def test_oracle_connectome_cross_connects_expected_regions():
    """test/test_tracking.py:227-253 on the oracle, with the region aggregation of tg.connectome."""
    from scipy.spatial import cKDTree

    fod, mask = data.cross()
    seg = data.cross_segmentation()
    domain, field = tg.domain.Image(mask), tg.field.Image(fod)
    alg = tg.algorithm.Transport(tg.local.RealSymmetricSphericalHarmonics(45), step_size=0.25, gamma=0.0)
    m = _oracle_matrix(alg, domain, field, 10000, 12.0)
    seg_data = np.asarray(seg.dataobj)
    labels = np.unique(seg_data[seg_data > 0])
    vox = np.argwhere(seg_data > 0)
    d, nearest = cKDTree(vox.astype(float)).query(domain.boundary.vertices, distance_upper_bound=2.0)
    ok = np.isfinite(d)
    lab = np.zeros(len(d), np.intp)
    hit = vox[nearest[ok]]
    lab[ok] = np.searchsorted(labels, seg_data[hit[:, 0], hit[:, 1], hit[:, 2]])
    sel = np.flatnonzero(ok)
    A = csr_matrix((np.ones(len(sel), np.float32), (lab[sel], sel)), shape=(len(labels), len(d)))
    region = (A @ m @ A.T).toarray()
    und = region + region.T
    for r, partner in enumerate([1, 0, 3, 2]):
        assert und[r, partner] > np.delete(und[r], [r, partner]).max()


def test_connectome_validation():
    domain = tg.domain.Image(tg.Nifti1Image(np.ones((1, 1, 1), np.uint8), np.eye(4)))
    field = tg.field.Image(tg.Nifti1Image(np.zeros((1, 1, 1, 15), np.float32), np.eye(4)))
    alg = tg.algorithm.Transport(tg.local.RealSymmetricSphericalHarmonics(15))
    with pytest.raises(ValueError):
        tg.tracking.connectome(alg, domain, field, n_seeds=-1)
    with pytest.raises(ValueError):
        tg.tracking.connectome(alg, domain, field, n_seeds=1, maximum_streamline_length=1.0,
                               minimum_streamline_length=2.0)
    with pytest.raises(ValueError):
        tg.connectome(field, 1, distance_upper_bound=-1.0)
    m, labels = tg.connectome(field, 1, domain, alg, tg.Nifti1Image(np.zeros((1, 1, 1), np.uint8), np.eye(4)))
    assert m.shape == (0, 0) and len(labels) == 0
