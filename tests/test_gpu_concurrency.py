"""Trackers used concurrently: two jobs in flight on two streams.

Each runtime owns a stream, a tracker and its own device copies of the
field and domain; trackers share no state, and the C ABI's error message is
per host thread.  Two host threads each run a sequence of tg_tracker_run
calls on their own runtime, so that one job's tracking overlaps the other's
(as bench.py does with two jobs in flight).  Every result must equal, bit
for bit, the same job run alone.
"""

import threading

import numpy as np
import pytest

import tractography_b200 as tg

from helpers import bits_equal, small_config0

pytestmark = pytest.mark.gpu


def _job(field, domain, seeds, k):
    model = tg.local.RealSymmetricSphericalHarmonics(45)
    if k % 2:
        alg = tg.algorithm.Diffusion(model, step_size=0.05, gamma=1.0, noise_variance=0.1, seed=k)
    else:
        alg = tg.algorithm.Transport(model, step_size=0.2, gamma=1.0)
    rng = np.array([1000 + 31 * k + b for b in range(4)], np.uint32)
    return alg, rng


def test_two_jobs_in_flight_equal_jobs_alone(runtime):
    import torch

    field, domain, seeds = small_config0(n_voxels=16, n_seeds=2000, seed=11)
    n_jobs = 6
    batch = 500
    alone = []
    for k in range(n_jobs):
        alg, rng = _job(field, domain, seeds, k)
        alone.append(tg.tracking.track_packed(alg, domain, field, seeds, save_at=0.25, n_steps=80,
                                              batch_size=batch, batch_rng_seeds=rng, runtime=runtime))
    slots = [tg.CudaRuntime(runtime.device, stream=torch.cuda.Stream(runtime.device)) for _ in range(2)]
    got = [None] * n_jobs
    errors = []

    def worker(w):
        try:
            rt = slots[w]
            with rt.device_scope():
                for k in range(w, n_jobs, 2):
                    alg, rng = _job(field, domain, seeds, k)
                    got[k] = tg.tracking.track_packed(alg, domain, field, seeds, save_at=0.25, n_steps=80,
                                                      batch_size=batch, batch_rng_seeds=rng, runtime=rt)
        except Exception as exc:  # reported after both threads end
            errors.append(exc)

    threads = [threading.Thread(target=worker, args=(w,)) for w in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for k in range(n_jobs):
        assert np.array_equal(got[k].lengths, alone[k].lengths), k
        assert bits_equal(got[k].points, alone[k].points), k
        assert got[k].steps == alone[k].steps, k
