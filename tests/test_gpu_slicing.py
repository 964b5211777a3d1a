"""Time slicing of the persistent tracker (tg_tracker_set_slicing).

A streamline whose saved points reach a multiple of the slice (slice_steps
in points: the largest power of two whose points take at most slice_steps
steps) while other work waits is saved to a device queue and resumed later
by whichever lane takes it.  Slices far shorter than the streamlines force
thousands of saves and resumes per run (with 2-step slices, one point per
slice: hundreds of thousands, so that the queue's slots are reused several
times); every result must still equal the oracle's, bit for bit, and the
run without slicing.  Covered: the SH image path (Diffusion and
Transport), the tensor closed-surface path, slicing together with tail
compaction, and slicing across retry waves of a point pool that is too
small.
"""

import ctypes

import numpy as np
import pytest

import tractography_b200 as tg
from tractography_b200 import _lib

from helpers import bits_equal, oracle_case, small_config0

pytestmark = pytest.mark.gpu


def _sh_job(kind, seed=3):
    model = tg.local.RealSymmetricSphericalHarmonics(45)
    if kind == "diffusion":
        return tg.algorithm.Diffusion(model, step_size=0.05, gamma=1.0, noise_variance=0.2, seed=seed)
    return tg.algorithm.Transport(model, step_size=0.05, gamma=1.0)


def _run(runtime, alg, domain, field, seeds, n_steps, batch=700):
    rng = np.array([1000 + 17 * b for b in range((len(seeds) + batch - 1) // batch)], np.uint32)
    return tg.tracking.track_packed(alg, domain, field, seeds, save_at=0.25, n_steps=n_steps, batch_size=batch,
                                    batch_rng_seeds=rng, runtime=runtime), rng


def _check_oracle(res, rng, alg, domain, field, seeds, n_steps, batch=700):
    for b, r in enumerate(rng):
        lo, hi = b * batch, min(len(seeds), (b + 1) * batch)
        want, want_len = oracle_case(alg, domain, field, rng_seed=int(r), save_at=0.25,
                                     n_steps=n_steps).tractogram(seeds[lo:hi], n_threads=8)
        assert np.array_equal(res.lengths[lo:hi], want_len), b
        for i in range(hi - lo):
            got = res.points[res.offsets[lo + i]: res.offsets[lo + i] + res.lengths[lo + i]]
            assert bits_equal(got, want[i, : want_len[i], :3]), (b, i)


def _stats(runtime):
    kms, waves, launches = ctypes.c_float(), ctypes.c_uint32(), ctypes.c_uint32()
    _lib.check(runtime.lib.tg_tracker_stats(runtime.tracker(), ctypes.byref(kms), ctypes.byref(waves),
                                            ctypes.byref(launches)))
    return waves.value


@pytest.mark.parametrize("kind,slice_steps,n_seeds", [("diffusion", 16, 2100), ("diffusion", 256, 2100),
                                                      ("transport", 64, 2100), ("diffusion", 2, 6300)])
def test_sliced_runs_equal_the_oracle_and_the_unsliced_run(kind, slice_steps, n_seeds):
    field, domain, seeds = small_config0(n_voxels=16, n_seeds=n_seeds, seed=8)
    n_steps = 120
    plain_rt = tg.CudaRuntime()
    plain_rt.set_slicing(0)
    plain, rng = _run(plain_rt, _sh_job(kind), domain, field, seeds, n_steps)
    rt = tg.CudaRuntime()
    rt.set_slicing(slice_steps)
    assert rt.slicing() == slice_steps
    sliced, _ = _run(rt, _sh_job(kind), domain, field, seeds, n_steps)
    assert np.array_equal(sliced.lengths, plain.lengths)
    assert np.array_equal(sliced.offsets, plain.offsets)
    assert bits_equal(sliced.points, plain.points)
    assert sliced.steps == plain.steps
    # streamlines run several slices each (~300 steps, ~60 points on
    # average); with one-point slices the queue's ~380k saves reuse its slots
    # several times over (its capacity is the seeds plus the launch's lanes)
    assert plain.steps / len(seeds) > 4 * min(slice_steps, 64)
    _check_oracle(sliced, rng, _sh_job(kind), domain, field, seeds, n_steps)


def test_slicing_with_tail_compaction():
    field, domain, seeds = small_config0(n_voxels=16, n_seeds=2100, seed=9)
    plain, rng = _run(tg.CudaRuntime(), _sh_job("diffusion", 5), domain, field, seeds, 100)
    rt = tg.CudaRuntime()
    rt.set_slicing(32)
    rt.set_tuning(0, 24, 3)
    both, _ = _run(rt, _sh_job("diffusion", 5), domain, field, seeds, 100)
    assert np.array_equal(both.lengths, plain.lengths)
    assert bits_equal(both.points, plain.points)
    assert both.steps == plain.steps


def test_slicing_across_retry_waves():
    field, domain, seeds = small_config0(n_voxels=16, n_seeds=1400, seed=10)
    plain, rng = _run(tg.CudaRuntime(), _sh_job("diffusion", 7), domain, field, seeds, 100)
    rt = tg.CudaRuntime(pool_points=8192)          # far below the points produced: several waves
    rt.set_slicing(16)
    waved, _ = _run(rt, _sh_job("diffusion", 7), domain, field, seeds, 100)
    assert _stats(rt) > 1
    assert np.array_equal(waved.lengths, plain.lengths)
    # a retried streamline is packed after the earlier waves' streamlines
    for i in range(len(seeds)):
        got = waved.points[waved.offsets[i]: waved.offsets[i] + waved.lengths[i]]
        want = plain.points[plain.offsets[i]: plain.offsets[i] + plain.lengths[i]]
        assert bits_equal(got, want), i


def test_sliced_closed_surface_run_equals_the_oracle():
    from tractography_b200 import synthetic

    fod = synthetic.dti_field(shape=(24, 24, 16), seed=2)
    v, f = synthetic.config2_surface(shape=(24, 24, 16), frequency=20)
    mesh = tg.domain.Mesh(v, f)
    field = tg.field.Image(fod)
    rt0 = tg.CudaRuntime()
    seeds = synthetic.seeds_inside(lambda p: tg.domain.contains(mesh, p, rt0), v.min(axis=0), v.max(axis=0), 1400,
                                   seed=4)
    alg = lambda: tg.algorithm.Diffusion(tg.local.DiffusionTensorImaging(), step_size=0.2, gamma=1.0,  # noqa: E731
                                         noise_variance=0.1, seed=6)
    plain, rng = _run(rt0, alg(), mesh, field, seeds, 160)
    rt = tg.CudaRuntime()
    rt.set_slicing(8)
    sliced, _ = _run(rt, alg(), mesh, field, seeds, 160)
    assert np.array_equal(sliced.lengths, plain.lengths)
    assert bits_equal(sliced.points, plain.points)
    assert plain.steps / len(seeds) > 3 * 8
    _check_oracle(sliced, rng, alg(), mesh, field, seeds, 160)


def test_slice_steps_must_be_a_power_of_two():
    rt = tg.CudaRuntime()
    assert rt.slicing() == 65536
    for bad in (3, 100, (1 << 30) + 1, 1 << 31):
        with pytest.raises(ValueError):
            rt.set_slicing(bad)
    rt.set_slicing(0)
    assert rt.slicing() == 0
