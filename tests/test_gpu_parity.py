"""CUDA path vs the CPU oracle, through the C ABI.

The kernels and the oracle perform the same IEEE binary32 operations in the
same order, so every comparison here is bit-exact (NaN equal to NaN): no
floating-point tolerance is used.  Config-0 Transport at a 0.1-voxel step is
chaotic (a 1e-7 perturbation grows to whole voxels), so agreement at any
tolerance looser than exact would not be reproducible over full lengths.
"""

import ctypes

import numpy as np
import pytest

import tractography_b200 as tg
from tractography_b200 import _lib

from helpers import bits_equal, oracle_case, random_orientations, small_config0

pytestmark = pytest.mark.gpu


def _device_rng_stream(runtime, which, state, n, maximum=0):
    import torch

    dtype = torch.int32 if which == 2 else torch.float32
    out = runtime.empty((n,), dtype)
    _lib.check(runtime.lib.tg_rng_stream(which, int(state[0]), int(state[1]), n, maximum,
                                         ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(runtime.stream_handle)))
    arr = out.cpu().numpy()
    return arr.view(np.uint32) if which == 2 else arr


@pytest.mark.parametrize("state", [(10, 4000), (1, 0), (123456789, 98765)])
def test_rng_streams_bit_exact(runtime, oracle, state):
    n = 4096
    assert bits_equal(_device_rng_stream(runtime, 0, state, n), oracle.randu_stream(state, n))
    assert bits_equal(_device_rng_stream(runtime, 1, state, n), oracle.randn_stream(state, n))
    assert np.array_equal(_device_rng_stream(runtime, 2, state, n, 100), oracle.randi_stream(state, n, 100))


@pytest.mark.parametrize("C", [1, 6, 15, 28, 45, 10])
def test_sh_local_evaluate_bit_exact(runtime, oracle, C):
    rng = np.random.default_rng(C)
    n = 3000
    o = random_orientations(rng, n)
    params = rng.normal(size=(n, C)).astype(np.float32)
    params[: n // 2, 0] += 3.0            # half in the linear softplus branch
    model = tg.local.RealSymmetricSphericalHarmonics(C)
    got = tg.local.evaluate(model, params, o, runtime)
    want = oracle.local_evaluate(oracle.MODEL_SH, params, o)
    assert bits_equal(got, want)


def test_dti_local_evaluate_bit_exact(runtime, oracle):
    rng = np.random.default_rng(5)
    n = 2000
    o = random_orientations(rng, n) * rng.uniform(0.5, 2.0, (n, 1)).astype(np.float32)
    params = rng.normal(size=(n, 6)).astype(np.float32)
    got = tg.local.evaluate(tg.local.DiffusionTensorImaging(), params, o, runtime)
    assert bits_equal(got, oracle.local_evaluate(oracle.MODEL_DTI, params, o))


@pytest.mark.parametrize("kind", ["transport", "diffusion", "diffusion_philox", "diffusion_zero_noise"])
@pytest.mark.parametrize("C", [6, 15, 45])
def test_update_orientation_bit_exact(runtime, oracle, kind, C):
    rng = np.random.default_rng(C + 17)
    n = 2000
    o = random_orientations(rng, n)
    params = rng.normal(size=(n, C)).astype(np.float32) * 0.2
    params[:, 0] += 1.0
    model = tg.local.DiffusionTensorImaging() if C == 6 else tg.local.RealSymmetricSphericalHarmonics(C)
    if C == 6:
        params = np.abs(params)
    if kind == "transport":
        alg = tg.algorithm.Transport(model, step_size=0.05, gamma=1.3)
    else:
        alg = tg.algorithm.Diffusion(model, step_size=0.05, gamma=1.3,
                                     noise_variance=0.0 if kind == "diffusion_zero_noise" else 0.3,
                                     seed=99, rng="philox" if kind == "diffusion_philox" else "mwc64x")
    twin_rng = np.random.default_rng(99)
    rng_seed = int(twin_rng.integers(0, np.iinfo(np.uint32).max, dtype=np.uint32)) if kind != "transport" else 0
    key = int(twin_rng.integers(0, 2 ** 63 - 1, dtype=np.int64)) if kind == "diffusion_philox" else 0
    got = tg.algorithm.update_orientation(alg, params, o, runtime)
    case = oracle.Case(model=oracle.MODEL_DTI if C == 6 else oracle.MODEL_SH,
                       algorithm=alg.algorithm_id, step_size=alg.step_size, gamma=alg.gamma,
                       noise_variance=getattr(alg, "noise_variance", 0.0), rng_mode=alg.rng_mode(),
                       rng_seed=rng_seed, philox_key=key)
    want = case.update_orientation(params, o)
    assert bits_equal(got, want)


def test_contains_and_field_evaluate_bit_exact(runtime, oracle):
    field, domain, _ = small_config0(n_voxels=12)
    rng = np.random.default_rng(3)
    pts = rng.uniform(-4, 30, size=(5000, 3)).astype(np.float32)
    pts[:8] = [[-1.0, 0, 0], [0.99, 1.0, 1.0], [1.0, 1.0, 1.0], [3.0, 3.0, 3.0], [5.0, 5.0, 5.0],
               [23.0, 23.0, 23.0], [-0.999, 0.0, 0.0], [22.999, 0, 0]]
    case = oracle_case(tg.algorithm.Transport(tg.local.RealSymmetricSphericalHarmonics(45)), domain, field)
    assert np.array_equal(tg.domain.contains(domain, pts, runtime), case.contains(pts))
    assert bits_equal(tg.field.evaluate(field, pts, runtime), case.field_evaluate(pts))


def _algorithms(model):
    return {
        "transport": lambda: tg.algorithm.Transport(model, step_size=0.2, gamma=1.0),
        "diffusion": lambda: tg.algorithm.Diffusion(model, step_size=0.05, gamma=1.0, noise_variance=0.1, seed=5),
        "philox": lambda: tg.algorithm.Diffusion(model, step_size=0.05, gamma=1.0, noise_variance=0.1, seed=5,
                                                 rng="philox"),
    }


@pytest.mark.parametrize("kind", ["transport", "diffusion", "philox"])
def test_tractogram_dense_and_packed_bit_exact(runtime, oracle, kind):
    field, domain, seeds = small_config0(n_voxels=16, n_seeds=300)
    make = _algorithms(tg.local.RealSymmetricSphericalHarmonics(45))[kind]
    n_steps = 80
    # dense (reference layout, one thread per seed) vs oracle
    alg = make()
    rng_seed, key = 2024, 0x1234_5678_9ABC
    dense, lengths = tg.tracking.tractogram_dense(alg, domain, field, seeds, save_at=0.25,
                                                  maximum_streamline_length=n_steps * 0.25, runtime=runtime,
                                                  rng_seed=rng_seed, philox_key=key)
    case = oracle_case(alg, domain, field, rng_seed=rng_seed, save_at=0.25, n_steps=n_steps, philox_key=key)
    want, want_len = case.tractogram(seeds)
    assert np.array_equal(lengths, want_len)
    for i in range(len(seeds)):
        assert bits_equal(dense[i, : lengths[i]], want[i, : want_len[i]]), i
    assert lengths.min() >= 1 and lengths.max() > 1

    # packed persistent tracker through the public low-level API, which draws
    # the call's seed (and key) from the algorithm as the reference does
    alg2, twin = make(), make()
    result = tg.tracking.tractogram(alg2, domain, field, seeds, save_at=0.25,
                                    maximum_streamline_length=n_steps * 0.25, runtime=runtime)
    rng_seed2 = twin.get_rng_seed()
    key2 = twin.philox_key() if kind == "philox" else 0
    case2 = oracle_case(alg2, domain, field, rng_seed=rng_seed2, save_at=0.25, n_steps=n_steps, philox_key=key2)
    want2, want_len2 = case2.tractogram(seeds)
    assert len(result.streamlines) == len(seeds)
    for i, s in enumerate(result.streamlines):
        assert bits_equal(s, want2[i, : want_len2[i], :3]), i


def test_tractogram_dti_bit_exact(runtime, oracle):
    from tractography_b200 import synthetic

    fod = synthetic.dti_field(shape=(20, 20, 12))
    field = tg.field.Image(fod)
    domain = tg.domain.Image(tg.Nifti1Image(np.ones(fod.shape[:3], np.uint8), fod.affine))
    seeds = synthetic.seeds_in_mask(tg.Nifti1Image(np.ones(fod.shape[:3], np.uint8), fod.affine), 200, seed=2)
    alg = tg.algorithm.Transport(tg.local.DiffusionTensorImaging(), step_size=0.2, gamma=5.0)
    result = tg.tracking.tractogram(alg, domain, field, seeds, save_at=0.5, maximum_streamline_length=30.0,
                                    runtime=runtime)
    case = oracle_case(alg, domain, field, save_at=0.5, n_steps=60)
    want, want_len = case.tractogram(seeds)
    for i, s in enumerate(result.streamlines):
        assert bits_equal(s, want[i, : want_len[i], :3]), i


def test_batches_keep_reference_streams(runtime, oracle):
    """tg.tractogram with batches == per-batch oracle calls with per-batch seeds."""
    field, domain, seeds = small_config0(n_voxels=16, n_seeds=250)
    model = tg.local.RealSymmetricSphericalHarmonics(45)
    alg = tg.algorithm.Diffusion(model, step_size=0.05, gamma=1.0, noise_variance=0.2, seed=11)
    twin = tg.algorithm.Diffusion(model, step_size=0.05, gamma=1.0, noise_variance=0.2, seed=11)
    fod_img = tg.Nifti1Image(field.values, np.linalg.inv(field.inverse_affine))
    result = tg.tractogram(fod_img, seeds, tg.Nifti1Image(domain.values, np.linalg.inv(domain.inverse_affine)),
                           alg, save_at=0.25, maximum_streamline_length=10.0, batch_size=100, runtime=runtime)
    got = list(result.streamlines)
    k = 0
    for start in range(0, len(seeds), 100):
        case = oracle_case(alg, domain, field, rng_seed=twin.get_rng_seed(), save_at=0.25, n_steps=40)
        want, want_len = case.tractogram(seeds[start:start + 100])
        for i in range(len(want_len)):
            assert bits_equal(got[k], want[i, : want_len[i], :3]), (start, i)
            k += 1
    assert k == len(got)


@pytest.mark.parametrize("model", ["sh", "dti"])
def test_seeds_from_fod_bit_exact(runtime, oracle, model):
    from tractography_b200 import synthetic

    if model == "sh":
        fod, _ = synthetic.config0(n=10)
        mid = oracle.MODEL_SH
    else:
        fod = synthetic.dti_field(shape=(10, 10, 6))
        mid = oracle.MODEL_DTI
    inline, voxels, affine = tg.seeds.sparse_fod(fod)
    states = np.random.default_rng(4).integers(0, 2 ** 32 - 1, size=(3000, 2), dtype=np.uint32)
    got = tg.seeds.seeds_from_sparse_fod(mid, inline, voxels, affine, states, runtime)
    want = oracle.seeds_from_fod(mid, inline, voxels, affine, states)
    assert bits_equal(got, want)
    assert np.allclose(np.linalg.norm(got[:, 4:7], axis=1), 1, atol=1e-5)
    assert np.all(got[:, 3] == 1) and np.all(got[:, 7] == 0)
