"""Many jobs in one device-scheduled run (tg_tracker_run_jobs) vs the oracle, bit for bit.

Jobs differ in model (SH lmax 2/4/6/8, tensor), algorithm, grid, length
budget, batch size and seed count; each job's streamlines must equal the
oracle's per-batch results exactly (same RNG seed per batch, stream id =
index in batch).  A tiny point pool forces several retry waves, which must
not change any result.
"""

import numpy as np
import pytest

import tractography_b200 as tg
from tractography_b200 import jobs as jobs_module
from tractography_b200 import synthetic

from helpers import bits_equal, oracle_case

pytestmark = pytest.mark.gpu


def make_jobs():
    rng = np.random.default_rng(9)
    out = []
    specs = [((12, 12, 12), 8, "transport", 300, 40, 100),
             ((10, 14, 9), 4, "diffusion", 257, 25, 64),
             ((12, 12, 12), 6, "diffusion", 90, 60, 1000),
             ((9, 9, 9), 2, "transport", 33, 15, 7),
             ("dti", 0, "diffusion", 150, 30, 50),
             ((16, 16, 16), 8, "diffusion", 500, 50, 128),
             ((12, 12, 12), 8, "transport", 0, 10, 10)]
    for shape, lmax, kind, n, n_steps, batch in specs:
        if shape == "dti":
            fod = synthetic.dti_field(shape=(14, 14, 10), seed=4)
            mask = tg.Nifti1Image(np.ones(fod.shape[:3], np.uint8), fod.affine)
            model = tg.local.DiffusionTensorImaging()
            step = 0.3
        else:
            fod, mask = synthetic.bundle_field(shape, lmax=lmax, seed=int(rng.integers(100)))
            model = tg.local.RealSymmetricSphericalHarmonics((lmax + 1) * (lmax + 2) // 2)
            step = 0.2
        if kind == "transport":
            alg = tg.algorithm.Transport(model, step_size=step, gamma=1.0 if shape != "dti" else 5.0)
        else:
            alg = tg.algorithm.Diffusion(model, step_size=step, gamma=1.0, noise_variance=0.15,
                                         seed=int(rng.integers(1000)))
        seeds = synthetic.uniform_seeds(mask, n, seed=int(rng.integers(1000))) if n else np.empty((0, 8), np.float32)
        n_batches = max(1, (n + batch - 1) // batch) if n else 0
        rng_seeds = np.array([alg.get_rng_seed() for _ in range(n_batches)], dtype=np.uint32)
        out.append(jobs_module.Job(field=tg.field.Image(fod), domain=tg.domain.Image(mask), algorithm=alg,
                                   seeds=seeds, save_at=0.25, n_steps=n_steps, min_points=0, batch_size=batch,
                                   batch_rng_seeds=rng_seeds))
    return out


def check_against_oracle(jobs, result):
    for j, job in enumerate(jobs):
        r = result.job(j)
        assert len(r.lengths) == job.n_seeds
        for b, rng_seed in enumerate(job.batch_rng_seeds):
            lo, hi = b * job.batch_size, min(job.n_seeds, (b + 1) * job.batch_size)
            case = oracle_case(job.algorithm, job.domain, job.field, rng_seed=int(rng_seed), save_at=job.save_at,
                               n_steps=job.n_steps)
            want, want_len = case.tractogram(job.seeds[lo:hi])
            assert np.array_equal(r.lengths[lo:hi], want_len), (j, b)
            seq = r.streamlines()
            for i in range(hi - lo):
                assert bits_equal(seq[lo + i], want[i, : want_len[i], :3]), (j, b, i)


@pytest.mark.parametrize("tuning", [(0, 0, 4), (0, 8, 4), (2, 31, 2), (0, 24, 16)])
def test_run_jobs_bit_exact(tuning):
    runtime = tg.CudaRuntime()
    runtime.set_tuning(*tuning)
    jobs = make_jobs()
    result = jobs_module.run_jobs_packed(jobs, runtime)
    assert result.steps > 0
    check_against_oracle(jobs, result)


@pytest.mark.parametrize("tuning", [(0, 0, 0), (1, 31, 3), (0, 16, 16)])
def test_single_job_tuning_does_not_change_results(tuning):
    """tg_tracker_run with any launch shape and tail compaction equals the oracle."""
    from helpers import small_config0

    field, domain, seeds = small_config0(n_voxels=16, n_seeds=3000, seed=5)
    alg = tg.algorithm.Diffusion(tg.local.RealSymmetricSphericalHarmonics(45), step_size=0.1, gamma=1.0,
                                 noise_variance=0.2, seed=3)
    twin = tg.algorithm.Diffusion(tg.local.RealSymmetricSphericalHarmonics(45), step_size=0.1, gamma=1.0,
                                  noise_variance=0.2, seed=3)
    runtime = tg.CudaRuntime()
    runtime.set_tuning(*tuning)
    assert runtime.tuning() == dict(zip(("blocks_per_sm", "compact_lanes", "compact_rounds"), tuning))
    result = tg.tracking.tractogram(alg, domain, field, seeds, save_at=0.25, maximum_streamline_length=40.0,
                                    runtime=runtime)
    want, want_len = oracle_case(alg, domain, field, rng_seed=twin.get_rng_seed(), save_at=0.25,
                                 n_steps=160).tractogram(seeds, n_threads=8)
    for i, s in enumerate(result.streamlines):
        assert bits_equal(s, want[i, : want_len[i], :3]), i


def test_run_jobs_with_retry_waves_bit_exact():
    runtime = tg.CudaRuntime(pool_points=4096)     # far below the points produced: forces waves
    jobs = make_jobs()
    result = jobs_module.run_jobs_packed(jobs, runtime)
    import ctypes

    kms, waves, launches = ctypes.c_float(), ctypes.c_uint32(), ctypes.c_uint32()
    runtime.lib.tg_tracker_stats(runtime.tracker(), ctypes.byref(kms), ctypes.byref(waves), ctypes.byref(launches))
    assert waves.value > 1
    check_against_oracle(jobs, result)


def test_run_jobs_returns_tractograms_like_tractogram(runtime):
    jobs = make_jobs()[:3]
    together = jobs_module.run_jobs(jobs, runtime)
    for job, t in zip(jobs, together):
        alone = jobs_module.run(job, runtime)
        assert len(alone.streamlines) == len(t.streamlines)
        for a, b in zip(alone.streamlines, t.streamlines):
            assert bits_equal(a, b)
