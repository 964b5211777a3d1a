"""The oracle against the reference's own kernels compiled for the CPU (oracle/_ref).

oracle/build_ref.py builds libtgref.so from the OpenCL source the reference
assembles itself (build() runs it where the reference tree is present).
These tests pin the oracle -- and through the bit-exact GPU tests, the CUDA
path -- to the reference kernel:

* known answers of the reference's tests on the reference kernel;
* Diffusion with the reference's MWC64X noise stream: point-wise within
  1e-4 voxel over the first 100 steps for >= 99.9 % of seeds, identical
  lengths;
* non-chaotic Transport cases (exact u0u3 solution, circle): point-wise;
* chaotic config-0 Transport (step 0.1 voxel): single-step float32 error of
  the oracle against the reference's float64 NumPy update no larger than the
  reference kernel's own, and the length distributions of the two agree
  (two-sample KS test).
"""

import numpy as np
import pytest

import tractography_b200 as tg
from oracle import oracle as O
from oracle import reference as R
from tractography_b200 import synthetic

import data
from helpers import oracle_case

pytestmark = pytest.mark.skipif(not R.available(), reason="oracle/_ref not built (reference sources absent)")


def test_reference_kernel_known_answers():
    """test/test_tracking.py:28-100 on the reference kernel itself."""
    f = np.zeros((1, 1, 1, 15), np.float32)
    f[..., 0] = 1.0
    s = np.array([[0, 0, 0, 1, 1, 0, 0, 0]], np.float32)
    out, n, _ = R.tractogram_raw(np.ones((1, 1, 1)), np.eye(4), f, np.eye(4), "sh", "transport", 1.0, 0.0, 0.0, 0,
                                 s, 1.0, 300)
    np.testing.assert_allclose(out[0, : n[0], :3], [[0, 0, 0], [1, 0, 0]], atol=1e-6)
    f = np.zeros((20, 1, 1, 15), np.float32)
    f[..., 0] = 1.0
    out, n, _ = R.tractogram_raw(np.ones((20, 1, 1)), np.eye(4), f, np.eye(4), "sh", "transport", 0.25, 0.0, 0.0,
                                 0, s, 0.5, 6)
    np.testing.assert_allclose(out[0, :6, 0], np.arange(0.0, 3.0, 0.5), atol=1e-6)


def test_diffusion_first_100_steps_match_reference_kernel():
    fod, mask = synthetic.bundle_field((48, 56, 48), lmax=8, seed=3, voxel_mm=1.25)
    field = tg.field.Image(fod)
    domain = tg.domain.Image(tg.Nifti1Image(np.any(field.values != 0, -1).astype(np.uint8), fod.affine))
    seeds = synthetic.uniform_seeds(mask, 4000, seed=1)
    alg = tg.algorithm.Diffusion(tg.local.RealSymmetricSphericalHarmonics(45), step_size=0.001, gamma=1.0,
                                 noise_variance=0.1, seed=0)
    ref, ref_len, _ = R.tractogram(domain, field, alg, seeds, 12345, 0.001, 101, threads=8)
    got, got_len = oracle_case(alg, domain, field, rng_seed=12345, save_at=0.001, n_steps=101).tractogram(
        seeds, n_threads=8)
    assert np.array_equal(ref_len, got_len)
    deviation = np.abs(ref[:, :, :3] - got[:, :, :3]).max(axis=(1, 2)) / 1.25      # voxels
    assert np.mean(deviation <= 1e-4) >= 0.999


@pytest.mark.parametrize("algorithm", ["transport", "diffusion"])
def test_u0u3_matches_reference_kernel(algorithm):
    coef = data.u0u3_coefficients(0.3, 45)
    f = np.broadcast_to(coef, (1, 1, 1, 45)).astype(np.float32).copy()
    A = np.diag((1000.0, 1000.0, 1000.0, 1.0))
    A[:3, 3] = -0.5
    inv = np.linalg.inv(A).astype(np.float32)
    o = np.asarray(tg.core.sph2cart(0.5, 0.12, 1.0))
    s = np.array([[10, 10, 10, 1, *o, 0]], np.float32)
    ref, ref_len, _ = R.tractogram_raw(np.ones((1, 1, 1)), inv, f, inv, "sh", algorithm, 0.001, 1.0, 0.0, 5, s,
                                       0.001, 1000)
    case = O.Case(mask=np.ones((1, 1, 1)), mask_inv_affine=inv, field=f, field_inv_affine=inv,
                  algorithm=O.ALGO_TRANSPORT if algorithm == "transport" else O.ALGO_DIFFUSION, step_size=0.001,
                  gamma=1.0, noise_variance=0.0, rng_seed=5, save_at=0.001, n_steps=1000)
    got, got_len = case.tractogram(s)
    assert np.array_equal(ref_len, got_len)
    np.testing.assert_allclose(got[0, : got_len[0], :3], ref[0, : ref_len[0], :3], atol=1e-4)


def test_circle_matches_reference_kernel():
    fod = data.circle(shape=(10, 10, 1), radius=2).astype(np.float32)
    wm = fod[..., 0] > 0
    s = np.array([[4.5, 6.5, 0.0, 1.0, 1.0, 0.0, 0.0, 0.0]], np.float32)
    ref, ref_len, _ = R.tractogram_raw(wm, np.eye(4), fod, np.eye(4), "sh", "transport", 1e-4, 50.0, 0.0, 0, s,
                                       0.25, 400)
    got, got_len = O.Case(mask=wm, mask_inv_affine=np.eye(4), field=fod, field_inv_affine=np.eye(4),
                          step_size=1e-4, gamma=50.0, save_at=0.25, n_steps=400).tractogram(s)
    assert ref_len[0] == got_len[0] == 400
    np.testing.assert_allclose(got[0, :400, :3], ref[0, :400, :3], atol=1e-4)


def test_config0_transport_single_step_and_length_distribution():
    from scipy.stats import ks_2samp

    fod, mask = synthetic.config0()
    field = tg.field.Image(fod)
    domain = tg.domain.Image(mask)
    seeds = synthetic.seeds_in_mask(mask, 2000, seed=0)
    params = field.evaluate(seeds[:, :3])
    o = seeds[:, 4:7]
    alg = tg.algorithm.Transport(tg.local.RealSymmetricSphericalHarmonics(45), step_size=0.2, gamma=1.0)
    exact = alg.update_orientation(params.astype(np.float64), o.astype(np.float64))
    ref1 = R.update_orientation("sh", 45, "transport", 0.2, 1.0, 0.0, 0, params, o)
    got1 = O.Case(algorithm=O.ALGO_TRANSPORT, step_size=0.2, gamma=1.0).update_orientation(params, o)
    err_ref = np.median(np.abs(ref1 - exact).max(axis=1))
    err_got = np.median(np.abs(got1 - exact).max(axis=1))
    assert err_got <= 1.2 * err_ref
    ref, ref_len, _ = R.tractogram(domain, field, alg, seeds, 0, 0.25, 1200, threads=8)
    got, got_len = oracle_case(alg, domain, field, save_at=0.25, n_steps=1200).tractogram(seeds, n_threads=8)
    assert ks_2samp(ref_len, got_len).pvalue > 0.01
    ends_ref = ref[np.arange(len(seeds)), ref_len - 1, :3]
    ends_got = got[np.arange(len(seeds)), got_len - 1, :3]
    for axis in range(3):
        assert ks_2samp(ends_ref[:, axis], ends_got[:, axis]).pvalue > 0.01


@pytest.mark.parametrize("name", ["sphere", "voxels"])
def test_boundary_seeds_match_reference_kernel(name):
    """domain.seed's sampler: the oracle equals the reference kernel bit for bit."""
    from pathlib import Path

    G = np.load(Path(__file__).resolve().parent / "golden" / "bvh_reference.npz")
    args = (G[f"{name}_vertices"], G[f"{name}_triangles"], G[f"{name}_cumulative"])
    for rng_seed in (0, 12345, 0xFFFFFFFF):
        want = R.boundary_seeds(*args, rng_seed, 3000)
        got = O.boundary_seeds(*args, rng_seed, 3000)
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def _cross_case():
    import data as _data

    fod, mask = _data.cross(shape=(12, 12, 3))
    field, domain = tg.field.Image(fod), tg.domain.Image(mask)
    b = domain.boundary_bvh()
    return field, domain, O.BoundaryBvh.build(b.vertices, b.faces)


@pytest.mark.parametrize("gamma", [0.0, 1.0])
def test_tod_transport_matches_reference_kernel(gamma):
    """tracking.py:255-356 (the reference's own tod kernel) vs the oracle: sums agree to float tolerance."""
    field, domain, bvh = _cross_case()
    alg = tg.algorithm.Transport(tg.local.RealSymmetricSphericalHarmonics(45), step_size=0.1, gamma=gamma)
    ref = R.tod(domain, field, bvh, "transport", 0.1, gamma, 0.0, 99, 3000, 80, (12, 12, 3), np.eye(4), threads=8)
    got = oracle_case(alg, domain, field, rng_seed=99).tod(domain.boundary_arrays(), 3000, 80, (12, 12, 3),
                                                           np.eye(4))
    assert np.abs(ref - got).sum() <= 1e-4 * np.abs(ref).sum()


def test_connectome_transport_matches_reference_kernel():
    """tracking.py:458-553: same start/end vertices for >= 99.9 % of tracks, weights to float tolerance."""
    field, domain, bvh = _cross_case()
    alg = tg.algorithm.Transport(tg.local.RealSymmetricSphericalHarmonics(45), step_size=0.1, gamma=1.0)
    r2, c2, w2 = R.connectome(domain, field, bvh, "transport", 0.1, 1.0, 0.0, 99, 20000, 120, 0.5, threads=8)
    r1, c1, w1 = oracle_case(alg, domain, field, rng_seed=99).connectome(bvh, domain.boundary_arrays(), 20000, 120,
                                                                         0.5)
    assert np.mean(r1 == r2) >= 0.999
    same = (r1 == r2) & (r1 >= 0)
    assert np.mean((c1 == c2)[same] & (np.abs(w1 - w2)[same] <= 1e-4)) >= 0.999


def test_diffusion_tod_and_connectome_within_reference_sampling_noise():
    """With noise the tracks diverge between any two binary32 implementations (ill-conditioned drift);
    the distance of the oracle's result from the reference's is below that of two reference runs
    with different seeds."""
    from tractography_b200.tracking import contributions_to_matrix

    field, domain, bvh = _cross_case()
    alg = tg.algorithm.Diffusion(tg.local.RealSymmetricSphericalHarmonics(45), step_size=0.1, gamma=1.0,
                                 noise_variance=0.05)
    nv = len(domain.boundary.vertices)
    case = oracle_case(alg, domain, field, rng_seed=99)

    def mat(r):
        return contributions_to_matrix(*r, nv).toarray()

    A = mat(R.connectome(domain, field, bvh, "diffusion", 0.1, 1.0, 0.05, 99, 20000, 120, 0.5, threads=8))
    B = mat(R.connectome(domain, field, bvh, "diffusion", 0.1, 1.0, 0.05, 100, 20000, 120, 0.5, threads=8))
    C = mat(case.connectome(bvh, domain.boundary_arrays(), 20000, 120, 0.5))
    assert np.abs(A - C).sum() < np.abs(A - B).sum()
    T1 = R.tod(domain, field, bvh, "diffusion", 0.1, 1.0, 0.05, 99, 20000, 80, (12, 12, 3), np.eye(4), threads=8)
    T2 = R.tod(domain, field, bvh, "diffusion", 0.1, 1.0, 0.05, 100, 20000, 80, (12, 12, 3), np.eye(4), threads=8)
    T3 = case.tod(domain.boundary_arrays(), 20000, 80, (12, 12, 3), np.eye(4))
    assert np.abs(T1 - T3).sum() < np.abs(T1 - T2).sum()


@pytest.mark.parametrize("model", ["sh", "dti"])
def test_fod_seeding_matches_reference_kernel(model):
    """seeds.from_fod (seeds.py:174-216) on the reference's own seeds.cl kernel vs
    the oracle, on identical MWC64X states drawn as the reference draws them
    (np.random.randint(4294967295, size=(n, 2)), seeds.py:185).

    * voxel choice and jitter (seeds.cl:89-94) are integer and exact float
      arithmetic: the world locations agree bit for bit for every seed;
    * the orientation is the first of 1000 Fibonacci directions whose
      cumulative softplus'd model value exceeds a uniform threshold
      (seeds.cl:29-56).  The same direction is chosen for >= 99.9 % of seeds,
      and where one differs it is the neighbouring direction in the
      cumulative order (the sums round differently at the threshold);
    * the chosen directions agree to 2.4e-7 (the reference's sincos/sqrt come
      from the platform's libm, the oracle's from tg_fmath.h).

    The GPU tests then pin the CUDA seeding to the oracle bit for bit."""
    if model == "sh":
        fod, _ = synthetic.config0(n=16)
    else:
        fod = synthetic.dti_field(shape=(24, 24, 16), seed=4)
    inline, voxels, affine = tg.seeds.sparse_fod(fod)
    states = np.random.RandomState(11).randint(4294967295, size=(4000, 2)).astype(np.uint32)
    ref, ref_states = R.seeds_from_fod(model, inline, voxels, affine, states, threads=4)
    ours = O.seeds_from_fod(O.MODEL_DTI if model == "dti" else O.MODEL_SH, inline, voxels, affine, states,
                            n_threads=4)
    assert np.array_equal(ref[:, :4].view(np.uint32), ours[:, :4].view(np.uint32))
    assert np.all(ref[:, 7] == 0.0) and np.all(ours[:, 7] == 0.0)
    fib = synthetic.fibonacci(1000)
    i_ref = np.argmax(ref[:, 4:7] @ fib.T, axis=1)
    i_ours = np.argmax(ours[:, 4:7] @ fib.T, axis=1)
    same = i_ref == i_ours
    assert same.mean() >= 0.999, same.mean()
    assert np.all(np.abs(i_ref[~same] - i_ours[~same]) == 1), (i_ref[~same], i_ours[~same])
    assert np.abs(ref[same, 4:7] - ours[same, 4:7]).max() <= 2.4e-7
    # the kernel writes back the states after its draws (seeds.cl:117)
    assert not np.array_equal(ref_states, states)
