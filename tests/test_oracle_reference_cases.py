"""The reference test suite's known answers, checked on the CPU oracle.

Each test restates a case of the reference's own tests (cited per test) and
runs it through the oracle, pinning the oracle to the reference's expected
behaviour.  The GPU tests then check the CUDA path against the oracle.
"""

import numpy as np
import pytest

import tractography_b200 as tg
from oracle import oracle as O

import data

EYE = np.eye(4)


def case(mask, field, **kw):
    mask = np.asarray(mask)
    return O.Case(mask=mask, mask_inv_affine=kw.pop("mask_inv", EYE), field=field,
                  field_inv_affine=kw.pop("field_inv", EYE), **kw)


def seed(x, y, z, dx, dy, dz):
    return np.array([[x, y, z, 1.0, dx, dy, dz, 0.0]], dtype=np.float32)


def test_tracks_seed_until_leaving_domain():
    """test/test_tracking.py:28-53"""
    f = np.zeros((1, 1, 1, 15), np.float32)
    f[..., 0] = 1.0
    out, n = case(np.ones((1, 1, 1)), f, step_size=1.0, gamma=0.0, save_at=1.0, n_steps=300).tractogram(
        seed(0, 0, 0, 1, 0, 0))
    np.testing.assert_allclose(out[0, : n[0], :3], [[0, 0, 0], [1, 0, 0]], atol=1e-6)


def test_save_interval_and_maximum_length():
    """test/test_tracking.py:71-100: 6 points at x = 0, 0.5, ..., 2.5."""
    f = np.zeros((20, 1, 1, 15), np.float32)
    f[..., 0] = 1.0
    out, n = case(np.ones((20, 1, 1)), f, step_size=0.25, gamma=0.0, save_at=0.5, n_steps=6).tractogram(
        seed(0, 0, 0, 1, 0, 0))
    assert n[0] == 6
    np.testing.assert_allclose(out[0, :6, 0], np.arange(0.0, 3.0, 0.5), atol=1e-6)
    np.testing.assert_allclose(out[0, :6, 1:3], 0.0, atol=1e-6)


def test_diffusion_without_noise_is_deterministic():
    """test/test_tracking.py:103-127"""
    f = np.zeros((1, 1, 1, 15), np.float32)
    f[..., 0] = 1.0
    out, n = case(np.ones((1, 1, 1)), f, algorithm=O.ALGO_DIFFUSION, step_size=1.0, gamma=0.0, noise_variance=0.0,
                  rng_seed=1234, save_at=1.0, n_steps=300).tractogram(seed(0, 0, 0, 1, 0, 0))
    np.testing.assert_allclose(out[0, : n[0], :3], [[0, 0, 0], [1, 0, 0]], atol=1e-6)


@pytest.mark.parametrize("algorithm", [O.ALGO_TRANSPORT, O.ALGO_DIFFUSION])
def test_u0u3_exact_solution(algorithm):
    """test/test_algorithms/test_transport.py:28-144 and test_diffusion.py:15-71 (zero noise)."""
    eps, C = 0.3, 45
    coef = data.u0u3_coefficients(eps, C)
    f = np.broadcast_to(coef, (1, 1, 1, C)).astype(np.float32).copy()
    affine = np.diag((1000.0, 1000.0, 1000.0, 1.0))
    affine[:3, 3] = -0.5
    inv = np.linalg.inv(affine)
    theta0, phi0 = 0.12, 0.5
    o = np.asarray(tg.core.sph2cart(phi0, theta0, 1.0))
    c = case(np.ones((1, 1, 1)), f, mask_inv=inv, field_inv=inv, algorithm=algorithm, step_size=0.001, gamma=1.0,
             noise_variance=0.0, rng_seed=5, save_at=0.001, n_steps=1000)
    out, n = c.tractogram(seed(10, 10, 10, *o))
    line = out[0, : n[0], :3].astype(np.float64)
    u = data.u0u3_reference(0.001, 1.0, theta0, phi0, eps, len(line))
    expected = np.empty_like(line)
    expected[0] = [10, 10, 10]
    for k in range(1, len(line)):
        expected[k] = expected[k - 1] + 0.001 * u[k]
    np.testing.assert_array_almost_equal(line, expected, decimal=3)


def test_transport_circle_runs_to_maximum_length():
    """test/test_algorithms/test_transport.py:209-239 (step 1e-4, gamma 50, 100 mm)."""
    shape, radius = (10, 10, 1), 2
    fod = data.circle(shape=shape, radius=radius).astype(np.float32)
    wm = fod[..., 0] > 0
    s = seed((shape[0] - 1) / 2, (shape[1] - 1) / 2 + radius, 0.0, 1.0, 0.0, 0.0)
    c = case(wm, fod, step_size=1e-4, gamma=50.0, save_at=0.25, n_steps=400)
    out, n = c.tractogram(s)
    assert n[0] * 0.25 == pytest.approx(100.0)


def test_diffusion_circle_runs_to_maximum_length():
    """test/test_algorithms/test_diffusion.py:153-189 (100 seeds, noise 0.1)."""
    shape, radius = (10, 10, 1), 2
    fod = data.circle(shape=shape, radius=radius).astype(np.float32)
    wm = fod[..., 0] > 0
    s = np.repeat(seed((shape[0] - 1) / 2, (shape[1] - 1) / 2 + radius, 0.0, 1.0, 0.0, 0.0), 100, axis=0)
    c = case(wm, fod, algorithm=O.ALGO_DIFFUSION, step_size=1e-3, gamma=50.0, noise_variance=0.1, rng_seed=99,
             save_at=0.25, n_steps=400)
    out, n = c.tractogram(s, n_threads=8)
    assert np.all(n * 0.25 == pytest.approx(100.0))


def test_tensor_circle_runs_to_maximum_length():
    """test/test_algorithms/test_diffusion.py:127-151 (DTI, 10 seeds, 40 mm)."""
    tensors, wm = data.tensor_circle((20, 20, 1), radius=5, width=2)
    field = tg.field.Image(tensors)
    domain = tg.domain.Image(tg.Nifti1Image(np.any(field.values != 0, -1).astype(np.uint8), tensors.affine))
    s = np.repeat(seed(19.0, 22.5, 0.0, -1.0, 0.0, 0.0), 10, axis=0)
    c = O.Case(mask=domain.values, mask_inv_affine=domain.inverse_affine, field=field.values,
               field_inv_affine=field.inverse_affine, model=O.MODEL_DTI, algorithm=O.ALGO_DIFFUSION,
               step_size=0.001, gamma=10.0, noise_variance=0.01, rng_seed=3, save_at=0.25, n_steps=160)
    out, n = c.tractogram(s, n_threads=8)
    assert np.all(n * 0.25 == pytest.approx(40.0))


def test_uniform_isotropic_streamlines_are_straight():
    """test/test_algorithms/test_transport.py:155-171 (|second difference| < 1e-3)."""
    fod = data.uniform_isotropic().astype(np.float32)
    np.random.seed(0)
    inline, voxels, affine = tg.seeds.sparse_fod(tg.Nifti1Image(fod, EYE))
    states = np.random.randint(4294967295, size=(40, 2)).astype(np.uint32)
    seeds = O.seeds_from_fod(O.MODEL_SH, inline, voxels, affine, states)
    c = case(np.any(fod != 0, -1), fod, step_size=0.001, gamma=0.5, save_at=0.25, n_steps=1200)
    out, n = c.tractogram(seeds, n_threads=8)
    for i in range(len(seeds)):
        d = np.diff(out[i, : n[i], :3], n=2, axis=0)
        assert np.all(d < 1e-3)


def test_cross_coverage_stays_in_mask():
    """test/test_algorithms/test_transport.py:173-190: points stay inside the cross (no coverage claim)."""
    fod, wm = data.cross()
    mask = wm.get_fdata().astype(np.uint8)
    fod_data = (fod.get_fdata() * mask[..., None]).astype(np.float32)
    np.random.seed(1)
    s = tg.seeds.from_mask(wm, 300)
    c = case(np.any(fod_data != 0, -1), fod_data, step_size=0.001, gamma=0.5, save_at=0.25, n_steps=1200)
    out, n = c.tractogram(s, n_threads=8)
    pts = np.vstack([out[i, : n[i] - 1, :3] for i in range(len(s)) if n[i] > 1])
    vox = np.round(pts).astype(int)
    assert np.all(mask[tuple(vox.T)] == 1)


def test_field_rounds_half_voxels_to_even():
    """test/test_field.py:20-33"""
    values = np.arange(64, dtype=np.float32).reshape(4, 4, 4, 1)
    pts = np.array([[0.5, 1.5, 2.5], [1.5, 0.5, 0.5], [-0.5, 2.5, 2.5]], np.float32)
    got = O.Case(field=values, field_inv_affine=EYE).field_evaluate(pts)
    np.testing.assert_array_equal(got, values[[0, 2, 0], [2, 0, 2], [2, 0, 2]])


def test_field_zero_outside_and_non_cubic_indexing():
    """test/test_field.py:8-18, 36-46"""
    values = np.arange(2 * 3 * 4 * 2, dtype=np.float32).reshape(2, 3, 4, 2)
    c = O.Case(field=values, field_inv_affine=EYE)
    pts = np.array([[0, 0, 0], [1, 2, 3], [1, 0, 2]], np.float32)
    np.testing.assert_array_equal(c.field_evaluate(pts), values[[0, 1, 1], [0, 2, 0], [0, 3, 2]])
    outside = np.array([[-0.51, 0, 0], [0, 3, 0], [0, 0, 4]], np.float32)
    np.testing.assert_array_equal(c.field_evaluate(outside), 0.0)


def test_contains_uses_half_open_cells_and_world_coordinates():
    """test/test_domain.py:133-145 and 34-48"""
    c = O.Case(mask=np.ones((1, 1, 1)), mask_inv_affine=EYE)
    pts = np.array([[-0.5, 0, 0], [0.49, 0.49, 0.49], [0.5, 0, 0]], np.float32)
    np.testing.assert_array_equal(c.contains(pts), [True, True, False])
    img = np.zeros((3, 3, 3))
    img[1, 1, 1] = 1
    affine = np.eye(4)
    affine[:3, 3] = (10, 20, 30)
    c2 = O.Case(mask=img, mask_inv_affine=np.linalg.inv(affine).astype(np.float32))
    np.testing.assert_array_equal(c2.contains(np.array([[11, 21, 31], [10, 20, 30]], np.float32)), [True, False])


def test_randu_and_randi_ranges():
    """test/test_src/test_utils.py:17-56 (state {10, 4000}, 1e6 values)."""
    u = O.randu_stream((10, 4000), 1_000_000)
    assert u.min() > 0 and u.max() < 1
    i = O.randi_stream((10, 4000), 1_000_000, 100)
    assert i.min() >= 0 and i.max() <= 99


def test_update_orientation_matches_analytic_step():
    """test/test_algorithm.py:54-74 and 77-103 (rtol/atol 2e-4 / 3e-4)."""
    def coefficients(base, eps, C=15):
        d = tg.core.fibonacci_sphere(1000)
        az, co, _ = tg.core.cart2sph(*d.T)
        Y, _ = tg.core.ishtmtx(az, co, C)
        return np.linalg.lstsq(Y, base + eps * d[:, 0] * d[:, 2], rcond=None)[0].astype(np.float32)

    def expected(o, base, eps, step, gamma):
        raw = base + eps * o[0] * o[2]
        value = np.logaddexp(0.0, 100.0 * raw) / 100.0
        d = 1.0 / (1.0 + np.exp(-100.0 * raw))
        g = eps * np.array([o[2], 0.0, o[0]])
        t = step * gamma * d / value * (g - o * np.dot(o, g))
        n = np.linalg.norm(t)
        return o.copy() if n == 0 else np.cos(n) * o + np.sin(n) / n * t

    fods = [(0.1, 0.2), (0.25, 0.4), (0.05, 0.55), (0.1, 0.3)]
    params = np.stack([coefficients(b, e) for b, e in fods])
    phi = np.array([0.3, 1.2, 2.4, 0.5])
    theta = np.array([0.6, 1.1, 2.0, 0.8])
    o = np.stack(tg.core.sph2cart(phi, theta, 1.0), -1)
    c = O.Case(algorithm=O.ALGO_TRANSPORT, step_size=0.025, gamma=1.3)
    got = c.update_orientation(params, o)
    want = np.stack([expected(o[i], *fods[i], 0.025, 1.3) for i in range(4)])
    np.testing.assert_allclose(got, want, rtol=3e-4, atol=3e-4)
    np.testing.assert_allclose(np.linalg.norm(got, axis=1), 1.0, atol=1e-5)


def test_update_orientation_finite_at_poles():
    """test/test_algorithm.py:133-150"""
    d = tg.core.fibonacci_sphere(1000)
    az, co, _ = tg.core.cart2sph(*d.T)
    Y, _ = tg.core.ishtmtx(az, co, 15)
    p = np.linalg.lstsq(Y, 0.1 + 0.3 * d[:, 0] * d[:, 2], rcond=None)[0].astype(np.float32)
    phi = np.array([0.0, 1.1, 0.7, 2.0])
    theta = np.array([0.0, np.pi, 1e-4, np.pi - 1e-4])
    o = np.stack(tg.core.sph2cart(phi, theta, 1.0), -1)
    got = O.Case(algorithm=O.ALGO_TRANSPORT, step_size=0.01, gamma=1.0).update_orientation(np.repeat(p[None], 4, 0), o)
    assert np.all(np.isfinite(got))
    np.testing.assert_allclose(np.linalg.norm(got, axis=1), 1.0, atol=1e-6)
    assert np.all(np.linalg.norm(got - o, axis=1) > 0.0)


def test_diffusion_update_is_seeded_and_normalised():
    """test/test_algorithm.py:185-202"""
    p = np.zeros((3, 15), np.float32)
    p[:, 0] = 1.0
    o = np.eye(3, dtype=np.float32)
    c = O.Case(algorithm=O.ALGO_DIFFUSION, step_size=0.001, gamma=1.0, noise_variance=1.0, rng_seed=1234)
    a, b = c.update_orientation(p, o), c.update_orientation(p, o)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_allclose(np.linalg.norm(a, axis=1), 1.0, atol=1e-5)
    assert np.any(np.linalg.norm(a - o, axis=1) > 0.0)


@pytest.mark.parametrize("kind", ["sh", "dti"])
def test_seed_orientations_follow_the_fod(kind):
    """test/test_seeds.py:163-213: second moment of 60000 seeds vs the density, atol 2e-2."""
    d = tg.core.fibonacci_sphere(1000)
    if kind == "sh":
        fod, _ = data.cross()
        coef = fod.get_fdata()[5, 1, 0]
        az, co, _ = tg.core.cart2sph(*d.T)
        Y, _ = tg.core.ishtmtx(az, co, 45)
        v = Y @ coef
        w = np.where(100 * v < 30, np.log1p(np.exp(np.clip(100 * v, -700, 30))) / 100, v)
        model, C = O.MODEL_SH, 45
    else:
        tensors, _ = data.tensor_cross()
        coef = tensors.get_fdata()[10, 1, 0]
        T = np.array([[coef[0], coef[3], coef[4]], [coef[3], coef[1], coef[5]], [coef[4], coef[5], coef[2]]])
        w = np.einsum("ni,ij,nj->n", d, T, d)
        model, C = O.MODEL_DTI, 6
    prob = np.maximum(w, 0)
    prob /= prob.sum()
    expected = np.einsum("n,ni,nj->ij", prob, d, d)
    states = np.random.default_rng(0).integers(0, 2 ** 32 - 1, size=(60000, 2), dtype=np.uint32)
    seeds = O.seeds_from_fod(model, coef[None].astype(np.float32), np.array([[0, 0, 0, 1]], np.float32),
                             np.eye(4, dtype=np.float32), states, n_threads=8)
    o = seeds[:, 4:7]
    np.testing.assert_allclose(np.einsum("ni,nj->ij", o, o) / len(o), expected, atol=2e-2)
    assert np.all(np.abs(seeds[:, :3]) <= 0.5)


def test_oracle_tractogram_ids_keys_streams_by_work_item():
    """A seed taken out of a larger call keeps that call's stream (rng_init(rng_seed, gid),
    core.cl:203-208): tractogram_ids on a subset equals the full call's rows."""
    from helpers import oracle_case, small_config0

    field, domain, seeds = small_config0(n_voxels=12, n_seeds=60, seed=4)
    alg = tg.algorithm.Diffusion(tg.local.RealSymmetricSphericalHarmonics(45), step_size=0.1, gamma=1.0,
                                 noise_variance=0.1, seed=3)
    c = oracle_case(alg, domain, field, rng_seed=99, save_at=0.25, n_steps=40)
    full, full_len = c.tractogram(seeds)
    ids = np.array([59, 3, 17, 40, 0], np.uint32)
    part, part_len = c.tractogram_ids(seeds[ids], ids)
    assert np.array_equal(part_len, full_len[ids])
    assert np.array_equal(part, full[ids], equal_nan=True)
    # the stream follows the id, not the position in the call
    other, _ = c.tractogram(seeds[ids])
    assert not np.array_equal(other, part, equal_nan=True)
