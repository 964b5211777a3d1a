"""Boundary connectome on the GPU vs the oracle, bit for bit (no atomics)."""

import numpy as np
import pytest

import tractography_b200 as tg
from oracle import oracle as O
from tractography_b200 import synthetic

import data
from helpers import oracle_case

pytestmark = pytest.mark.gpu


def _device_contributions(alg, domain, field, n_seeds, n_steps, min_len, runtime, rng_seed):
    import ctypes

    import torch
    from tractography_b200 import _lib, tracking
    from tractography_b200.algorithm import to_struct

    v4, f4, cum = domain.boundary_arrays()
    with runtime.device_scope():
        d_h, f_h = tracking._handles(alg, domain, field, runtime)
        b_h = domain.boundary_bvh().device(runtime)
        a = to_struct(alg, rng_seed)
        dv, df, dc = runtime.to_device(v4), runtime.to_device(f4), runtime.to_device(cum)
        rows = runtime.empty((9 * n_seeds,), torch.int32)
        cols = runtime.empty((9 * n_seeds,), torch.int32)
        w = runtime.empty((9 * n_seeds,), torch.float32)
        steps = torch.zeros((1,), dtype=torch.int64, device=runtime.device)
        _lib.check(runtime.lib.tg_connectome(
            ctypes.byref(a), d_h, f_h, b_h, ctypes.c_void_p(dv.data_ptr()), len(v4), ctypes.c_void_p(df.data_ptr()),
            ctypes.c_void_p(dc.data_ptr()), len(f4), n_seeds, n_steps, min_len, ctypes.c_void_p(rows.data_ptr()),
            ctypes.c_void_p(cols.data_ptr()), ctypes.c_void_p(w.data_ptr()), ctypes.c_void_p(steps.data_ptr()),
            ctypes.c_void_p(runtime.stream_handle)))
        # the step counter: every track takes at most n_steps steps, and some take steps
        assert 0 < int(steps.item()) <= n_seeds * n_steps
        return rows.cpu().numpy(), cols.cpu().numpy(), w.cpu().numpy()


@pytest.mark.parametrize("kind", ["transport", "diffusion", "mesh"])
def test_connectome_contributions_bit_exact(runtime, kind):
    fod, mask = data.cross(shape=(12, 12, 3))
    field = tg.field.Image(fod)
    model = tg.local.RealSymmetricSphericalHarmonics(45)
    if kind == "mesh":
        v, f = synthetic.geodesic_sphere(10)
        domain = tg.domain.Mesh(v * np.array([4.0, 4.0, 0.9]) + np.array([5.5, 5.5, 1.0]), f)
    else:
        domain = tg.domain.Image(mask)
    alg = tg.algorithm.Transport(model, step_size=0.1, gamma=1.0) if kind != "diffusion" else \
        tg.algorithm.Diffusion(model, step_size=0.1, gamma=1.0, noise_variance=0.05, seed=3)
    n_seeds, n_steps, min_len = 5000, 120, 0.5
    got = _device_contributions(alg, domain, field, n_seeds, n_steps, min_len, runtime, 99)
    boundary = domain.boundary_bvh()
    bvh = O.BoundaryBvh.build(boundary.vertices, boundary.faces)
    want = oracle_case(alg, domain, field, rng_seed=99).connectome(bvh, domain.boundary_arrays(), n_seeds, n_steps,
                                                                   min_len)
    assert np.array_equal(got[0], want[0])
    valid = want[0] >= 0
    assert np.array_equal(got[1][valid], want[1][valid])
    assert np.array_equal(got[2][valid].view(np.uint32), want[2][valid].view(np.uint32))
    assert 0.1 < valid.mean() <= 1.0


def test_tg_connectome_cross_regions(runtime):
    """test/test_tracking.py:227-253 through the public API."""
    fod, mask = data.cross()
    alg = tg.algorithm.Transport(tg.local.RealSymmetricSphericalHarmonics(45), step_size=0.25, gamma=0.0)
    matrix, labels = tg.connectome(fod, n_seeds=10000, domain=mask, algorithm=alg,
                                   segmentation=data.cross_segmentation(), distance_upper_bound=2.0,
                                   maximum_streamline_length=12.0, runtime=runtime)
    np.testing.assert_array_equal(labels, [1, 2, 3, 4])
    und = matrix + matrix.T
    for r, partner in enumerate([1, 0, 3, 2]):
        assert und[r, partner] > np.delete(und[r], [r, partner]).max()
    m = tg.tracking.connectome(alg, tg.domain.Image(mask), tg.field.Image(fod), n_seeds=16,
                               maximum_streamline_length=2.0, runtime=runtime)
    assert m.dtype == np.float32 and m.shape == (len(tg.domain.Image(mask).boundary.vertices),) * 2
