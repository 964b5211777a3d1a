"""Streaming tractogram files (tg.write_tractogram) on the GPU.

The file must hold exactly the streamlines tg.tractogram returns for the
same request, in the same order: seeds are tracked a few batches per pass,
and each batch keeps its own RNG seed and per-batch stream ids (MWC64X) or
its global seed index (Philox), so splitting into passes changes nothing.
"""

import numpy as np
import pytest

import tractography_b200 as tg
from tractography_b200 import synthetic

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("rng", ["mwc64x", "philox"])
@pytest.mark.parametrize("suffix", [".tck", ".trx"])
def test_write_tractogram_equals_tractogram(runtime, tmp_path, rng, suffix):
    fod, mask = synthetic.bundle_field((16, 16, 16), lmax=8, seed=5)
    seeds = synthetic.uniform_seeds(mask, 1000, seed=2)
    model = tg.local.RealSymmetricSphericalHarmonics(45)

    def algorithm():
        return tg.algorithm.Diffusion(model, step_size=0.2, gamma=1.0, noise_variance=0.1, seed=33, rng=rng)

    kw = dict(save_at=0.25, maximum_streamline_length=15.0, minimum_streamline_length=2.0, batch_size=96,
              runtime=runtime)
    want = tg.tractogram(fod, seeds, mask, algorithm(), **kw)
    path = tmp_path / f"out{suffix}"
    n = tg.write_tractogram(path, fod, seeds, mask, algorithm(), seeds_per_pass=250, **kw)
    assert n == len(want.streamlines) and 0 < n < len(seeds)
    got = tg.load_tck(path).streamlines if suffix == ".tck" else tg.load_trx(path)[0].streamlines
    assert len(got) == n
    for a, b in zip(want.streamlines, got):
        assert np.array_equal(np.asarray(a), np.asarray(b))
