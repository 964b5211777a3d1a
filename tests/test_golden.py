"""Oracle and host code vs golden vectors produced by the reference itself.

tests/golden/reference_numpy.npz holds outputs of the reference's own
float64 NumPy implementations (local.py, algorithm.py, field.py, domain.py,
core.py, seeds.py) on seeded inputs; tests/golden/make_golden.py regenerates
it from the reference sources.  Float32 kernels are compared with the
tolerance the reference's own tests use for its OpenCL-vs-NumPy checks
(1e-4, test/test_local.py:43, 68); integer and index results exactly.
"""

from pathlib import Path

import numpy as np
import pytest

import tractography_b200 as tg
from oracle import oracle as O

G = np.load(Path(__file__).resolve().parent / "golden" / "reference_numpy.npz")


@pytest.mark.parametrize("C", [15, 28, 45])
def test_sh_model_matches_reference(C):
    got = O.local_evaluate(O.MODEL_SH, G[f"sh{C}_params"], G[f"sh{C}_orient"])
    np.testing.assert_allclose(got, G[f"sh{C}_value"], rtol=1e-4, atol=1e-4)


def test_dti_model_matches_reference():
    got = O.local_evaluate(O.MODEL_DTI, G["dti_params"], G["dti_orient"])
    np.testing.assert_allclose(got, G["dti_value"], rtol=1e-4, atol=1e-8)


@pytest.mark.parametrize("name,algorithm,step,gamma", [
    ("transport", O.ALGO_TRANSPORT, 0.01, 1.5),
    ("diffusion0", O.ALGO_DIFFUSION, 0.02, 0.7),
])
def test_one_step_updates_match_reference(name, algorithm, step, gamma):
    c = O.Case(algorithm=algorithm, step_size=step, gamma=gamma, noise_variance=0.0)
    got = c.update_orientation(G["sh45_params"], G["sh45_orient"])
    np.testing.assert_allclose(got, G[f"{name}_update"], rtol=2e-4, atol=2e-4)


def test_dti_transport_update_matches_reference():
    c = O.Case(model=O.MODEL_DTI, algorithm=O.ALGO_TRANSPORT, step_size=0.1, gamma=10.0)
    got = c.update_orientation(G["dti_params"], G["dti_orient"])
    np.testing.assert_allclose(got, G["dti_transport_update"], rtol=2e-4, atol=2e-4)


def test_field_sampling_matches_reference_exactly():
    c = O.Case(field=G["field_img"], field_inv_affine=G["field_inv_affine"])
    np.testing.assert_array_equal(c.field_evaluate(G["field_points"]), G["field_value"])


def test_domain_membership_matches_reference_exactly():
    c = O.Case(mask=G["mask"], mask_inv_affine=G["mask_inv_affine"])
    np.testing.assert_array_equal(c.contains(G["mask_points"]), G["mask_contains"])
    d = tg.domain.Image(tg.Nifti1Image(G["mask"], G["affine"]))
    np.testing.assert_array_equal(d.contains(G["mask_points"]), G["mask_contains"])


def test_core_helpers_match_reference():
    Y, dY = tg.core.ishtmtx(G["ishtmtx_az"], G["ishtmtx_co"], 45)
    np.testing.assert_allclose(Y, G["ishtmtx_Y"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(dY, G["ishtmtx_dY"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(tg.core.fibonacci_sphere(1000), G["fibonacci1000"], rtol=0, atol=1e-15)
    np.testing.assert_allclose(np.stack(tg.core.cart2sph(*G["cart2sph_in"].T), -1), G["cart2sph_out"])


def test_numpy_model_methods_match_reference():
    for C in (15, 28, 45):
        got = tg.local.RealSymmetricSphericalHarmonics(C).evaluate(
            G[f"sh{C}_params"].astype(np.float64), G[f"sh{C}_orient"].astype(np.float64))
        np.testing.assert_allclose(got, G[f"sh{C}_value"], rtol=1e-12, atol=1e-12)
    alg = tg.algorithm.Transport(tg.local.RealSymmetricSphericalHarmonics(45), step_size=0.01, gamma=1.5)
    np.testing.assert_allclose(alg.update_orientation(G["sh45_params"].astype(np.float64),
                                                      G["sh45_orient"].astype(np.float64)),
                               G["transport_update"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(tg.algorithm.exps2(G["exps2_p"], G["exps2_x"], 1.0), G["exps2_out"], atol=1e-15)


def test_host_seeding_is_identical_to_reference():
    """seeds.from_mask and the NumPy from_fod path draw the same legacy RNG values."""
    np.random.seed(7)
    got = tg.seeds.from_mask(tg.Nifti1Image(G["from_mask_input"], G["affine"]), 300)
    np.testing.assert_array_equal(got, G["from_mask"])
    np.random.seed(11)
    got = tg.seeds.from_fod(tg.Nifti1Image(G["from_fod_input"], G["affine"]), 120, use_opencl=False)
    np.testing.assert_array_equal(got, G["from_fod_numpy"])
