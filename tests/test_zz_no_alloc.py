"""tg_tractogram_noalloc: tracking for callers that cannot let the library allocate.

Such callers -- a host application that owns the GPU memory budget and gives
plugins fixed buffers, or a loop that cannot afford cudaMalloc's possible
device synchronisation -- pass every input and output themselves; the only
scratch is the library's static device array.  This test calls the entry
point through the C ABI twice in a row (the array keeps the previous call's
contents, so the second call checks that the counters are cleared) and
compares both results with the existing entry points and the first batch
with the CPU oracle: bit for bit, the tolerance every parity test here
uses.  It lives in a file of its own that pytest collects last, and passes
alone in a fresh process or after the rest.
"""

import ctypes

import numpy as np
import pytest

import tractography_b200 as tg
from tractography_b200 import _lib
from tractography_b200.algorithm import to_struct

from helpers import bits_equal, oracle_case, small_config0

pytestmark = pytest.mark.gpu


def _noalloc(runtime, algorithm, domain, field, seeds, batch_size, rng_seeds, save_at, n_steps):
    import torch

    n = len(seeds)
    d_seeds = runtime.to_device(seeds)
    d_out = torch.zeros((n, n_steps, 4), dtype=torch.float32, device=runtime.device)
    d_len = torch.zeros((n,), dtype=torch.int32, device=runtime.device)
    rng = np.ascontiguousarray(rng_seeds, dtype=np.uint32)
    a = to_struct(algorithm)
    with runtime.device_scope():
        _lib.check(runtime.lib.tg_tractogram_noalloc(
            ctypes.byref(a), domain.device(runtime), field.device(runtime, _lib.MODEL_SH),
            ctypes.c_void_p(d_seeds.data_ptr()), n, batch_size, rng.ctypes.data_as(ctypes.c_void_p),
            float(save_at), n_steps, ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(d_len.data_ptr()),
            ctypes.c_void_p(runtime.stream_handle)))
        runtime.finish()
    return d_out.cpu().numpy(), d_len.cpu().numpy().view(np.uint32)


def test_noalloc_matches_existing_entry_points_twice():
    runtime = tg.CudaRuntime()
    field, domain, seeds = small_config0(n_voxels=16, n_seeds=400, seed=7)
    model = tg.local.RealSymmetricSphericalHarmonics(45)
    save_at, n_steps = 0.25, 60
    for call, (kind, batch_size) in enumerate([("diffusion", 150), ("transport", 400)]):
        if kind == "diffusion":
            alg = tg.algorithm.Diffusion(model, step_size=0.05, gamma=1.0, noise_variance=0.1, seed=call)
        else:
            alg = tg.algorithm.Transport(model, step_size=0.2, gamma=1.0)
        n_batches = (len(seeds) + batch_size - 1) // batch_size
        rng_seeds = np.array([1000 + 17 * b for b in range(n_batches)], dtype=np.uint32)
        out, lengths = _noalloc(runtime, alg, domain, field, seeds, batch_size, rng_seeds, save_at, n_steps)

        # existing dense entry point, one call per batch with that batch's seed
        for b in range(n_batches):
            sl = slice(b * batch_size, (b + 1) * batch_size)
            want, want_len = tg.tracking.tractogram_dense(alg, domain, field, seeds[sl], save_at=save_at,
                                                          maximum_streamline_length=n_steps * save_at,
                                                          runtime=runtime, rng_seed=int(rng_seeds[b]))
            assert np.array_equal(lengths[sl], want_len)
            for i in range(len(want_len)):
                assert bits_equal(out[sl][i, : want_len[i]], want[i, : want_len[i]]), (call, b, i)

        # and the CPU oracle for the first batch
        want, want_len = oracle_case(alg, domain, field, rng_seed=int(rng_seeds[0]), save_at=save_at,
                                     n_steps=n_steps).tractogram(seeds[:batch_size])
        assert np.array_equal(lengths[:batch_size], want_len)
        for i in range(len(want_len)):
            assert bits_equal(out[i, : want_len[i]], want[i, : want_len[i]]), (call, i)

        # existing persistent tracker over the same batches
        result = tg.tracking.track_packed(alg, domain, field, seeds, save_at=save_at, n_steps=n_steps,
                                          batch_size=batch_size, batch_rng_seeds=rng_seeds, runtime=runtime)
        assert np.array_equal(result.lengths, lengths)
        for i, s in enumerate(result.streamlines()):
            assert bits_equal(s, out[i, : lengths[i], :3]), (call, i)


def test_noalloc_rejects_too_many_batches():
    runtime = tg.CudaRuntime()
    field, domain, seeds = small_config0(n_voxels=12, n_seeds=20, seed=2)
    alg = tg.algorithm.Transport(tg.local.RealSymmetricSphericalHarmonics(45), step_size=0.2)
    n = 16385
    many = np.repeat(seeds[:1], n, axis=0)
    with pytest.raises(ValueError, match="exceed the maximum of 16384"):
        _noalloc(runtime, alg, domain, field, many, 1, np.zeros(n, np.uint32), 0.25, 4)
