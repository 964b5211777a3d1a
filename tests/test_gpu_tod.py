"""Track orientation distribution on the GPU vs the oracle.

The kernel sums each track's per-voxel run in order and adds it to the
output with atomicAdd, so voxels reached by several tracks sum in arbitrary
order: agreement with the oracle's sequential sum is to float tolerance
(relative 1e-5 of each voxel's largest coefficient), everything else (seeds,
tracks, voxel runs) being bit-identical.
"""

import numpy as np
import pytest

import tractography_b200 as tg
from tractography_b200 import synthetic

import data
from helpers import oracle_case

pytestmark = pytest.mark.gpu


def _compare(got, want):
    got, want = np.asarray(got, np.float64), np.asarray(want, np.float64)
    assert got.shape == want.shape
    scale = np.maximum(np.abs(want).max(axis=-1, keepdims=True), 1e-30)
    assert np.all(np.abs(got - want) <= 1e-5 * scale + 1e-7)
    assert np.array_equal(got[..., 0] != 0, want[..., 0] != 0)


@pytest.mark.parametrize("kind", ["transport", "diffusion", "mesh"])
def test_tod_matches_oracle(runtime, kind):
    fod, mask = data.cross(shape=(12, 12, 3))
    field = tg.field.Image(fod)
    model = tg.local.RealSymmetricSphericalHarmonics(45)
    if kind == "mesh":
        v, f = synthetic.geodesic_sphere(10)
        domain = tg.domain.Mesh(v * np.array([4.0, 4.0, 0.9]) + np.array([5.5, 5.5, 1.0]), f)
    else:
        domain = tg.domain.Image(mask)
    make = (lambda: tg.algorithm.Transport(model, step_size=0.1, gamma=1.0)) if kind == "transport" else \
        (lambda: tg.algorithm.Diffusion(model, step_size=0.1, gamma=1.0, noise_variance=0.05, seed=3))
    alg, twin = make(), make()
    stats = {}
    got = tg.tracking.tod(alg, domain, field, tg.Nifti1Image(np.zeros((12, 12, 3)), np.eye(4)), 3000,
                          maximum_streamline_length=8.0, runtime=runtime, stats=stats)
    raw = oracle_case(twin, domain, field, rng_seed=twin.get_rng_seed()).tod(
        domain.boundary_arrays(), 3000, 80, (12, 12, 3), np.eye(4))
    _compare(np.asarray(got.dataobj), tg.utils.normalize_odf(raw))
    assert np.count_nonzero(np.asarray(got.dataobj)[..., 0]) > 10
    # every accepted step inside the output grid added Y00 = 1 / (2 sqrt(pi)) to raw[..., 0]
    assert stats["steps"] <= 3000 * 80
    inside = float(raw[..., 0].sum(dtype=np.float64)) * 2.0 * np.sqrt(np.pi)   # float32 sums: to 1e-3
    assert stats["steps"] >= 0.999 * inside > 0


def test_tg_tod_reference_cases(runtime):
    """test/test_tractography.py:18-50."""
    fod, mask = data.cross()
    alg = tg.algorithm.Diffusion(tg.local.RealSymmetricSphericalHarmonics(45), step_size=0.01, gamma=1.0,
                                 noise_variance=0.1, seed=0)
    tod = tg.tod(fod, 32, mask, alg, maximum_streamline_length=20.0, runtime=runtime)
    d = np.asarray(tod.dataobj)
    assert tod.shape == fod.shape[:3] + (45,)
    assert np.isfinite(d).all()
    populated = d[..., 0] != 0
    assert np.any(populated)
    np.testing.assert_allclose(d[..., 0][populated], 1.0 / np.sqrt(4.0 * np.pi), rtol=1e-6)
    result = tg.tod(tg.field.Image(fod), n_seeds=16, maximum_streamline_length=2.0, runtime=runtime)
    assert result.shape == fod.shape[:3] + (45,)
