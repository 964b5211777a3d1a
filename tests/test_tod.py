"""Track orientation distribution: host logic and the oracle (reference tests' cases)."""

import numpy as np
import pytest

import tractography_b200 as tg
from oracle import oracle as O

from helpers import oracle_case


def test_tod_zero_seeds_returns_empty_image_without_gpu():
    """test/test_tracking.py:164-180."""
    desc = tg.Nifti1Image(np.zeros((2, 1, 1), np.float32), np.eye(4))
    dom = tg.domain.Image(tg.Nifti1Image(np.ones((1, 1, 1), np.uint8), np.eye(4)))
    field = tg.field.Image(tg.Nifti1Image(np.ones((1, 1, 1, 1), np.float32), np.eye(4)))
    alg = tg.algorithm.Transport(tg.local.RealSymmetricSphericalHarmonics(1))
    r = tg.tracking.tod(alg, dom, field, desc, n_seeds=0)
    assert r.shape == (2, 1, 1, 45)
    assert not np.any(np.asarray(r.dataobj))


def test_tod_validation():
    desc = tg.Nifti1Image(np.zeros((2, 1, 1), np.float32), np.eye(4))
    dom = tg.domain.Image(tg.Nifti1Image(np.ones((1, 1, 1), np.uint8), np.eye(4)))
    field = tg.field.Image(tg.Nifti1Image(np.ones((1, 1, 1, 1), np.float32), np.eye(4)))
    alg = tg.algorithm.Transport(tg.local.RealSymmetricSphericalHarmonics(1))
    with pytest.raises(ValueError):
        tg.tracking.tod(alg, dom, field, desc, n_seeds=-1)
    with pytest.raises(ValueError):
        tg.tracking.tod(alg, dom, field, desc, n_seeds=1, maximum_streamline_length=np.inf)
    with pytest.raises(ValueError):
        tg.tracking.tod(alg, dom, field, tg.Nifti1Image(np.zeros((2, 1)), np.eye(4)), n_seeds=1)
    with pytest.raises(ValueError):
        tg.tod(field, -1)
    with pytest.raises(TypeError):
        tg.tod(np.zeros((2, 2, 2, 15)), 1)


def test_oracle_tod_known_answer():
    """test/test_tracking.py:130-161 on the oracle: a populated voxel normalises to c0 = 1/sqrt(4 pi)."""
    f = np.zeros((1, 1, 1, 15), np.float32)
    f[..., 0] = 1.0
    field = tg.field.Image(tg.Nifti1Image(f, np.eye(4)))
    dom = tg.domain.Image(tg.Nifti1Image(np.ones((1, 1, 1), np.uint8), np.eye(4)))
    alg = tg.algorithm.Diffusion(tg.local.RealSymmetricSphericalHarmonics(15), step_size=0.1, gamma=0.0,
                                 noise_variance=0.0, seed=1234)
    raw = oracle_case(alg, dom, field, rng_seed=5).tod(dom.boundary_arrays(), 16, 3, (1, 1, 1), np.eye(4))
    tod = tg.utils.normalize_odf(raw)
    assert np.isfinite(tod).all()
    np.testing.assert_allclose(tod[0, 0, 0, 0], 1.0 / np.sqrt(4.0 * np.pi), atol=1e-6)
    # every seed deposits at least its first orientation
    assert raw[0, 0, 0, 0] >= 16 * 0.28209479 - 1e-4
