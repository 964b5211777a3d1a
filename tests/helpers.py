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
