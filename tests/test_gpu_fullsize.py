"""The CUDA tracker on the benchmarked workloads at full size.

Every other parity test runs on small volumes.  These run the two
workloads whose throughput the benchmark reports, with the benchmark's own
inputs (``synthetic.config1_workload`` / ``config2_workload``):

* the 145x174x145 lmax-8 Diffusion job, 1,000,000 seeds from
  ``seeds.from_fod`` in 20 batches of 50,000 (each batch with its own
  reference RNG seed and batch-local stream ids, 1200 points at most), run
  in one tg_tracker_run.  This reaches the paths a small volume does not:
  64-bit voxel offsets into the 702 MB padded field, domain and field on
  the same grid, stream ids up to 49,999;
* the 96x96x60 tensor field inside the ~499k-triangle closed surface,
  2,000,000 seeds, Transport at 0.1 voxel.

A spread sample of the seeds is tracked again by the CPU oracle (with each
seed's batch RNG seed and batch-local id, tracking.py:103-148) and must
match bit for bit: lengths and every point.  Size-independent properties
are checked over all seeds.
"""

import os

import numpy as np
import pytest

from tractography_b200 import synthetic

from helpers import bits_equal, oracle_case, tracker_run_sampled

pytestmark = pytest.mark.gpu

THREADS = os.cpu_count() or 1


def _check_sample(got, want, want_len, ids, label):
    for k, i in enumerate(ids):
        assert len(got[int(i)]) == want_len[k], (label, int(i), len(got[int(i)]), int(want_len[k]))
        assert bits_equal(got[int(i)], want[k, : want_len[k], :3]), (label, int(i))


def test_config1_full_size_matches_oracle_on_a_sample(runtime):
    n, batch, n_steps, save_at = 1_000_000, 50_000, 1200, 0.25
    fod, field, domain, seeds, alg = synthetic.config1_workload(n, runtime)
    n_batches = n // batch
    rng_seeds = np.array([alg.get_rng_seed() for _ in range(n_batches)], np.uint32)
    # 64 seeds per batch, spread over its stream ids (first and last included)
    local = np.unique(np.linspace(0, batch - 1, 64).astype(np.int64))
    sample = np.concatenate([b * batch + local for b in range(n_batches)])
    lengths, steps, total, got = tracker_run_sampled(runtime, alg, domain, field, seeds, save_at=save_at,
                                                     n_steps=n_steps, batch_size=batch, batch_rng_seeds=rng_seeds,
                                                     sample=sample)
    # size-independent properties over all seeds
    assert lengths.min() >= 1 and lengths.max() <= n_steps
    assert int(lengths.astype(np.int64).sum()) == total
    assert steps >= int((lengths.astype(np.int64) - 1).sum()) * 250   # 250 steps of 0.001 mm per 0.25 mm point
    for b in range(n_batches):
        ids = local
        case = oracle_case(alg, domain, field, rng_seed=int(rng_seeds[b]), save_at=save_at, n_steps=n_steps)
        want, want_len = case.tractogram_ids(seeds[b * batch + ids], ids, n_threads=THREADS)
        _check_sample(got, want, want_len, b * batch + ids, ("batch", b))
        assert all(bits_equal(got[int(b * batch + i)][0], seeds[b * batch + i, :3]) for i in ids)


def test_config2_full_size_matches_oracle_on_a_sample(runtime):
    n, n_steps, save_at = 2_000_000, 1200, 0.25
    field, mesh, seeds, alg = synthetic.config2_workload(n, runtime)
    assert len(mesh.faces) > 490_000
    sample = np.unique(np.linspace(0, n - 1, 2000).astype(np.int64))
    lengths, steps, total, got = tracker_run_sampled(runtime, alg, mesh, field, seeds, save_at=save_at,
                                                     n_steps=n_steps, batch_size=n, batch_rng_seeds=[0],
                                                     sample=sample)
    assert lengths.min() >= 1 and lengths.max() <= n_steps
    assert int(lengths.astype(np.int64).sum()) == total
    case = oracle_case(alg, mesh, field, rng_seed=0, save_at=save_at, n_steps=n_steps)
    want, want_len = case.tractogram_ids(seeds[sample], sample, n_threads=THREADS)
    _check_sample(got, want, want_len, sample, "config2")
    # streamlines of a Transport field stay in the surface for many steps
    assert np.median(lengths) > 10
