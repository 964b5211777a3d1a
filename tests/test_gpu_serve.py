"""Continuous-batching server: every request's result equals the job run alone.

Requests of several code paths (SH lmax 4/8, tensor; Transport and
Diffusion; image and mesh domains) arrive in waves while others run.  Short
epochs (by step count or by a device-clock deadline) force streamlines to be
carried across many epochs, and a small
point pool forces re-queued streamlines; neither may change a result: each
request must equal, bit for bit, the same job tracked alone by the packed
tracker (tg_tracker_run), and a few equal the CPU oracle directly.
"""

import numpy as np
import pytest

import tractography_b200 as tg
from tractography_b200 import jobs as jobs_module
from tractography_b200 import synthetic
from tractography_b200.serve import Server

from helpers import bits_equal, oracle_case

pytestmark = pytest.mark.gpu


def make_jobs(seed=0):
    rng = np.random.default_rng(seed)
    out = []
    fields = {}
    for k in range(12):
        kind = ["sh8", "sh4", "dti", "mesh"][k % 4]
        if kind == "dti" or kind == "mesh":
            fod = fields.setdefault("dti", synthetic.dti_field(shape=(24, 24, 16), seed=4))
            model = tg.local.DiffusionTensorImaging()
        else:
            lmax = 8 if kind == "sh8" else 4
            fod = fields.setdefault(kind, synthetic.bundle_field((14, 14, 14), lmax=lmax, seed=k)[0])
            model = tg.local.RealSymmetricSphericalHarmonics((lmax + 1) * (lmax + 2) // 2)
        field = tg.field.Image(fod)
        if kind == "mesh":
            v, f = synthetic.config2_surface(shape=(24, 24, 16), frequency=16)
            domain = fields.setdefault("mesh_domain", tg.domain.Mesh(v, f))
        else:
            domain = tg.domain.Image(tg.Nifti1Image(np.any(field.values != 0, -1).astype(np.uint8), fod.affine))
        mask = tg.Nifti1Image(np.ones(fod.shape[:3], np.uint8), fod.affine)
        n = int(rng.integers(50, 700))
        seeds = synthetic.uniform_seeds(mask, n, seed=int(rng.integers(1000)))
        if rng.uniform() < 0.5:
            alg = tg.algorithm.Transport(model, step_size=0.2, gamma=1.0)
        else:
            alg = tg.algorithm.Diffusion(model, step_size=0.2, gamma=1.0, noise_variance=0.1,
                                         seed=int(rng.integers(1000)))
        out.append(jobs_module.prepare(field, seeds, domain, alg, save_at=0.25,
                                       maximum_streamline_length=float(rng.uniform(10, 40)),
                                       batch_size=int(rng.integers(40, 300))))
    return out


def run_alone(job, runtime):
    return tg.tracking.track_packed(job.algorithm, job.domain, job.field, job.seeds, save_at=job.save_at,
                                    n_steps=job.n_steps, batch_size=job.batch_size,
                                    batch_rng_seeds=job.batch_rng_seeds, runtime=runtime,
                                    philox_key=job.philox_key)


@pytest.mark.parametrize("epoch_steps,pool_points,epoch_seconds",
                         [(1024, 0, 0.0), (7, 0, 0.0), (64, 6000, 0.0), (1 << 16, 0, 2e-5)])
def test_requests_equal_alone_in_the_mix(runtime, epoch_steps, pool_points, epoch_seconds):
    jobs = make_jobs()
    alone = [run_alone(j, runtime) for j in jobs]
    server = Server(runtime, hbm_budget_bytes=8e9, pool_points=pool_points, epoch_steps=epoch_steps,
                    max_requests=5, epoch_seconds=epoch_seconds)
    ids = {}
    results = {}
    waves = [jobs[:4], jobs[4:9], jobs[9:]]
    for w, wave in enumerate(waves):
        for j in wave:
            ids[server.submit(j)] = jobs.index(j)
        for _ in range(3 if w < 2 else 0):          # later waves arrive while earlier requests run
            for rid in server.poll():
                results[rid] = server.take(rid)
    polls = 0
    while len(results) < len(jobs):
        for rid in server.poll():
            results[rid] = server.take(rid)
        polls += 1
        assert polls < 20000, "requests stopped making progress"
    stats = server.stats()
    server.close()
    for rid, (points, offsets, lengths, seconds) in results.items():
        ref = alone[ids[rid]]
        assert np.array_equal(lengths, ref.lengths), rid
        for i in range(len(lengths)):
            a = points[offsets[i]:offsets[i] + lengths[i]]
            b = ref.points[ref.offsets[i]:ref.offsets[i] + ref.lengths[i]]
            assert bits_equal(a, b), (rid, i)
        assert len(points) == int(lengths.sum()) and seconds > 0
    # short epochs carry streamlines across many epochs
    assert stats.epochs >= (2 if epoch_steps >= 1024 else 20)
    assert stats.kernel_seconds > 0.0 and stats.harvest_seconds >= 0.0


def test_server_matches_oracle(runtime):
    job = make_jobs(seed=3)[1]
    with Server(runtime, hbm_budget_bytes=4e9, epoch_steps=13) as server:
        rid = server.submit(job)
        got = server.drain()[rid]
    n_batches = len(job.batch_rng_seeds)
    k = 0
    for b in range(n_batches):
        lo, hi = b * job.batch_size, min(job.n_seeds, (b + 1) * job.batch_size)
        want, want_len = oracle_case(job.algorithm, job.domain, job.field, rng_seed=int(job.batch_rng_seeds[b]),
                                     save_at=job.save_at, n_steps=job.n_steps).tractogram(job.seeds[lo:hi])
        for i in range(hi - lo):
            assert bits_equal(got.streamlines[k], want[i, : want_len[i], :3])
            k += 1
    assert k == len(got.streamlines)


def test_results_spanning_several_segments(runtime):
    """A request that saves far more points per seed than the server's
    admission estimate gets its result in several segments (new ones start
    without copying); the points taken back equal the job run alone."""
    fod, mask = synthetic.bundle_field((14, 14, 14), lmax=8, seed=2)
    seeds = synthetic.uniform_seeds(mask, 400, seed=9)
    model = tg.local.RealSymmetricSphericalHarmonics(45)
    alg = tg.algorithm.Diffusion(model, step_size=0.2, gamma=1.0, noise_variance=0.1, seed=5)
    job = jobs_module.prepare(tg.field.Image(fod), seeds, tg.domain.Image(mask), alg, save_at=0.05,
                              maximum_streamline_length=40.0, batch_size=128)
    alone = run_alone(job, runtime)
    assert alone.lengths.mean() > 160          # beyond the admission estimate of 160 points per seed
    with Server(runtime, hbm_budget_bytes=4e9, epoch_steps=9) as server:
        rid = server.submit(job)
        results = {}
        polls = 0
        while rid not in results:
            for r in server.poll():
                results[r] = server.take(r)
            polls += 1
            assert polls < 20000
        assert server.stats().epochs > 10
    points, offsets, lengths, _ = results[rid]
    assert np.array_equal(lengths, alone.lengths)
    for i in range(len(lengths)):
        assert bits_equal(points[offsets[i]:offsets[i] + lengths[i]],
                          alone.points[alone.offsets[i]:alone.offsets[i] + alone.lengths[i]]), i


def test_failed_reservation_only_warns(runtime):
    """A reservation larger than the device fails with a warning, and the
    server still serves: the failed allocation must not surface as the error
    of the next epoch's launch."""
    import torch

    total = torch.cuda.get_device_properties(runtime.device).total_memory
    job = make_jobs(seed=5)[0]
    alone = run_alone(job, runtime)
    with pytest.warns(UserWarning, match="reservation"):
        server = Server(runtime, hbm_budget_bytes=4e9, epoch_steps=64, reserve_bytes=2 * total)
    with server:
        rid = server.submit(job)
        got = server.drain()[rid]
    assert np.array_equal(np.array([len(s) for s in got.streamlines]), alone.lengths)
    for i, s in enumerate(got.streamlines):
        assert bits_equal(s, alone.points[alone.offsets[i]:alone.offsets[i] + alone.lengths[i]]), i
