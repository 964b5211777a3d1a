"""Helpers shared by the tests: oracle cases built from package objects."""

from __future__ import annotations

import numpy as np

import tractography_b200 as tg
from oracle import oracle as O


def oracle_case(algorithm, domain, field, *, rng_seed=0, save_at=1.0, n_steps=0, philox_key=0,
                seed_offset=0):
    model = O.MODEL_DTI if isinstance(algorithm.local_model, tg.local.DiffusionTensorImaging) else O.MODEL_SH
    algo = O.ALGO_DIFFUSION if isinstance(algorithm, tg.algorithm.Diffusion) else O.ALGO_TRANSPORT
    if isinstance(domain, tg.domain.Mesh):
        # the oracle's own BVH build of the same surface
        mask = dict(mesh=O.BoundaryBvh.build(domain.vertices, domain.faces))
    else:
        mask = dict(mask=domain.values, mask_inv_affine=domain.inverse_affine)
    return O.Case(
        **mask,
        field=field.values, field_inv_affine=field.inverse_affine,
        model=model, algorithm=algo, step_size=algorithm.step_size, gamma=algorithm.gamma,
        noise_variance=getattr(algorithm, "noise_variance", 0.0),
        rng_mode=algorithm.rng_mode(), rng_seed=rng_seed, philox_key=philox_key, seed_offset=seed_offset,
        save_at=save_at, n_steps=n_steps,
    )


def bits_equal(a, b) -> bool:
    """Equal shapes and identical float32 values (NaN equal to NaN)."""
    a = np.asarray(a, dtype=np.float32)
    b = np.asarray(b, dtype=np.float32)
    return a.shape == b.shape and bool(np.array_equal(a, b, equal_nan=True))


def random_orientations(rng, n, include_poles=True):
    phi = rng.uniform(0, 2 * np.pi, n)
    theta = np.arccos(rng.uniform(-1, 1, n))
    o = np.stack([np.sin(theta) * np.cos(phi), np.sin(theta) * np.sin(phi), np.cos(theta)], -1)
    if include_poles and n >= 6:
        o[:6] = [[0, 0, 1], [0, 0, -1], [1e-4, 0, 1], [0, -1e-4, -1], [1, 0, 0], [0.3, 0.4, 0.0]]
    return o.astype(np.float32)


def small_config0(n_voxels=16, n_seeds=200, seed=1):
    from tractography_b200 import synthetic

    fod, mask = synthetic.config0(n=n_voxels)
    seeds = synthetic.seeds_in_mask(mask, n_seeds, seed=seed)
    return tg.field.Image(fod), tg.domain.Image(mask), seeds


def tracker_run_sampled(runtime, algorithm, domain, field, seeds, *, save_at, n_steps, batch_size,
                        batch_rng_seeds, sample):
    """One tg_tracker_run over every seed (seeds resident on the device), then
    the points of the sampled seeds only.

    Returns (lengths of all seeds, accepted steps, total points, {seed: points})."""
    import ctypes

    from tractography_b200 import _lib
    from tractography_b200.algorithm import to_struct
    from tractography_b200.tracking import _handles

    n = int(seeds.shape[0])
    rng = np.ascontiguousarray(batch_rng_seeds, dtype=np.uint32)
    lengths = np.empty(n, np.uint32)
    offsets = np.empty(n, np.uint64)
    total, steps = ctypes.c_uint64(), ctypes.c_uint64()
    sh = ctypes.c_void_p(runtime.stream_handle)
    with runtime.device_scope():
        d_handle, f_handle = _handles(algorithm, domain, field, runtime)
        a = to_struct(algorithm)
        d_seeds = runtime.to_device(np.ascontiguousarray(seeds, np.float32))
        tracker = runtime.tracker()
        _lib.check(runtime.lib.tg_tracker_run(
            tracker, ctypes.byref(a), d_handle, f_handle, ctypes.c_void_p(d_seeds.data_ptr()), 0, n, int(batch_size),
            rng.ctypes.data_as(ctypes.c_void_p), float(save_at), int(n_steps), lengths.ctypes.data_as(ctypes.c_void_p),
            offsets.ctypes.data_as(ctypes.c_void_p), ctypes.byref(total), ctypes.byref(steps), sh))
        points = {}
        for i in sample:
            i = int(i)
            buf = np.zeros((int(lengths[i]), 3), np.float32)
            if len(buf):
                _lib.check(runtime.lib.tg_tracker_copy_points(tracker, buf.ctypes.data_as(ctypes.c_void_p),
                                                              int(offsets[i]), int(lengths[i]), 1, sh))
            points[i] = buf
        runtime.finish()
        del d_seeds
    return lengths, int(steps.value), int(total.value), points
