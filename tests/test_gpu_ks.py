"""Diffusion over 1M seeds: length and endpoint distributions vs the reference kernel.

The reference's own kernel source, compiled for the CPU (oracle/_ref), tracks
1M config-0 seeds with Diffusion in 50k-seed batches on the host cores; the
GPU tracks the same seeds (a) with the same per-batch MWC64X streams and (b)
with an independent Philox stream.  Point-wise agreement is not expected over
full lengths (the dynamics amplify binary32 rounding differences between any
two implementations); the distributions of streamline lengths and of each
endpoint coordinate must pass two-sample Kolmogorov-Smirnov tests.
"""

import os

import numpy as np
import pytest

import tractography_b200 as tg
from oracle import reference as R
from tractography_b200 import synthetic

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not R.available(), reason="oracle/_ref not built (reference sources absent)")]

N_SEEDS = 1_000_000
BATCH = 50_000
N_STEPS = 240          # 60 mm at save_at 0.25
P_MIN = 0.01


def _endpoints(points, offsets, lengths):
    return points[offsets + lengths - 1]


def test_diffusion_ks_1m_seeds(runtime):
    from scipy.stats import ks_2samp

    fod, mask = synthetic.config0()
    field, domain = tg.field.Image(fod), tg.domain.Image(mask)
    seeds = synthetic.seeds_in_mask(mask, N_SEEDS, seed=4)
    model = tg.local.RealSymmetricSphericalHarmonics(45)
    alg = tg.algorithm.Diffusion(model, step_size=0.2, gamma=1.0, noise_variance=0.1, seed=7)
    n_batches = N_SEEDS // BATCH
    rng = np.random.default_rng(5).integers(0, 2**32 - 1, n_batches, dtype=np.uint32)

    threads = os.cpu_count() or 1
    ref_len = np.empty(N_SEEDS, np.int64)
    ref_end = np.empty((N_SEEDS, 3), np.float32)
    for b in range(n_batches):
        lo, hi = b * BATCH, (b + 1) * BATCH
        out, L, _ = R.tractogram(domain, field, alg, seeds[lo:hi], int(rng[b]), 0.25, N_STEPS, threads=threads)
        ref_len[lo:hi] = L
        ref_end[lo:hi] = out[np.arange(BATCH), L.astype(np.int64) - 1, :3]

    same = tg.tracking.track_packed(alg, domain, field, seeds, save_at=0.25, n_steps=N_STEPS, batch_size=BATCH,
                                    batch_rng_seeds=rng, runtime=runtime)
    alg_p = tg.algorithm.Diffusion(model, step_size=0.2, gamma=1.0, noise_variance=0.1, seed=7, rng="philox")
    philox = tg.tracking.track_packed(alg_p, domain, field, seeds, save_at=0.25, n_steps=N_STEPS, batch_size=BATCH,
                                      batch_rng_seeds=rng, runtime=runtime, philox_key=alg_p.philox_key())
    assert 0.05 < np.mean(ref_len < N_STEPS) < 0.95
    for name, r in (("mwc64x", same), ("philox", philox)):
        end = _endpoints(r.points, r.offsets, r.lengths)
        assert ks_2samp(r.lengths, ref_len).pvalue > P_MIN, name
        for axis in range(3):
            assert ks_2samp(end[:, axis], ref_end[:, axis]).pvalue > P_MIN, (name, axis)
    # with the reference's noise stream most streamlines are identical in length
    assert np.mean(same.lengths == ref_len) > 0.5
