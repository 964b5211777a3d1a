"""Diffusion in the single-volume configuration: distributions vs the reference kernel.

The regime of the headline workload: the 145x174x145 lmax-8 volume at
1.25 mm, step 0.001 mm (about 1250 steps per voxel), gamma 1, noise
variance 0.1, seeds from seeds.from_fod (algorithm.py:198-228,
tracking.py:105-148).  Point-wise agreement is not expected over whole
streamlines: noise takes tracks into directions where the softplus'd model
value sits near its 1e-6 floor, and the drift divides by it, so any two
binary32 implementations part after some steps.  The distributions must
agree instead.

* the GPU tracks 1,000,000 seeds in 20 batches of 50,000 with the
  reference's per-batch MWC64X streams, and again with an independent
  Philox stream;
* the reference's own kernel source compiled for the CPU (oracle/_ref)
  tracks the first batch (50,000 seeds) on the host cores;
* the maximum length is 60 mm (240 points): a third of the streamlines
  leave the volume before it, and the reference sample costs about
  2.5e9 steps (about 45 s on 16 cores);
* the lengths and each endpoint coordinate pass two-sample
  Kolmogorov-Smirnov tests (p > 0.01) for both GPU runs.
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
N_REF = 50_000
N_STEPS = 240          # 60 mm at save_at 0.25
P_MIN = 0.01


def test_diffusion_ks_single_volume_regime(runtime):
    from scipy.stats import ks_2samp

    fod, field, domain, seeds, alg = synthetic.config1_workload(N_SEEDS, runtime)
    rng = np.array([alg.get_rng_seed() for _ in range(N_SEEDS // BATCH)], np.uint32)

    threads = os.cpu_count() or 1
    out, ref_len, _ = R.tractogram(domain, field, alg, seeds[:N_REF], int(rng[0]), 0.25, N_STEPS, threads=threads)
    ref_len = ref_len.astype(np.int64)
    ref_end = out[np.arange(N_REF), ref_len - 1, :3]
    del out
    assert 0.05 < np.mean(ref_len < N_STEPS) < 0.95

    same = tg.tracking.track_packed(alg, domain, field, seeds, save_at=0.25, n_steps=N_STEPS, batch_size=BATCH,
                                    batch_rng_seeds=rng, runtime=runtime)
    model = tg.local.RealSymmetricSphericalHarmonics(45)
    alg_p = tg.algorithm.Diffusion(model, step_size=0.001, gamma=1.0, noise_variance=0.1, seed=1234, rng="philox")
    philox = tg.tracking.track_packed(alg_p, domain, field, seeds, save_at=0.25, n_steps=N_STEPS, batch_size=BATCH,
                                      batch_rng_seeds=rng, runtime=runtime, philox_key=alg_p.philox_key())
    for name, r in (("mwc64x", same), ("philox", philox)):
        end = r.points[r.offsets + r.lengths - 1]
        assert ks_2samp(r.lengths, ref_len).pvalue > P_MIN, name
        for axis in range(3):
            assert ks_2samp(end[:, axis], ref_end[:, axis]).pvalue > P_MIN, (name, axis)
