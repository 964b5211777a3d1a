"""Host-side behaviour of the drop-in API (CPU only: validation, errors, containers, files).

Cases mirror the reference's tests for the same functions (cited per test).
None of these touch a GPU: empty inputs and invalid arguments are handled
before any device work, as in the reference.
"""

import numpy as np
import pytest

import tractography_b200 as tg


def sh_field(C=15, shape=(1, 1, 1), value=1.0):
    f = np.zeros(shape + (C,), dtype=np.float32)
    f[..., 0] = value
    return tg.field.Image(tg.Nifti1Image(f, np.eye(4)))


def test_empty_seeds_return_empty_tractogram():
    """test/test_tracking.py:10-25"""
    domain = tg.domain.Image(tg.Nifti1Image(np.ones((1, 1, 1)), np.eye(4)))
    field = tg.field.Image(tg.Nifti1Image(np.ones((1, 1, 1, 1)), np.eye(4)))
    alg = tg.algorithm.Transport(tg.local.RealSymmetricSphericalHarmonics(1))
    result = tg.tracking.tractogram(alg, domain, field, np.empty((0, 8), np.float32))
    assert len(result.streamlines) == 0
    np.testing.assert_array_equal(result.affine_to_rasmm, np.eye(4))


def test_incompatible_model_and_field():
    """test/test_tracking.py:56-68"""
    domain = tg.domain.Image(tg.Nifti1Image(np.ones((1, 1, 1)), np.eye(4)))
    field = tg.field.Image(tg.Nifti1Image(np.ones((1, 1, 1, 1)), np.eye(4)))
    alg = tg.algorithm.Transport(tg.local.RealSymmetricSphericalHarmonics(15))
    with pytest.raises(ValueError, match="15 != 1"):
        tg.tracking.tractogram(alg, domain, field, np.empty((0, 8), np.float32))


@pytest.mark.parametrize("kwargs,message", [
    ({"save_at": 0.0}, "save_at must be finite and positive."),
    ({"save_at": np.inf}, "save_at must be finite and positive."),
    ({"maximum_streamline_length": -1.0}, "maximum_streamline_length must be finite and non-negative."),
    ({"minimum_streamline_length": -1.0}, "minimum_streamline_length must be finite and non-negative."),
    ({"minimum_streamline_length": 5.0, "maximum_streamline_length": 1.0},
     "minimum_streamline_length must not exceed maximum_streamline_length."),
    ({"batch_size": 0}, "batch_size must be a positive integer."),
    ({"batch_size": 1.5}, "batch_size must be a positive integer."),
])
def test_tractogram_validates_numeric_options(kwargs, message):
    """tractography/__init__.py:433-444"""
    fod = tg.Nifti1Image(np.ones((2, 2, 2, 45), np.float32), np.eye(4))
    with pytest.raises(ValueError, match=message.replace(".", r"\.")):
        tg.tractogram(fod, np.empty((0, 8), np.float32), **kwargs)


def test_tractogram_type_errors():
    fod = tg.Nifti1Image(np.ones((2, 2, 2, 45), np.float32), np.eye(4))
    with pytest.raises(TypeError, match="field must be"):
        tg.tractogram("not a field", 3)
    with pytest.raises(TypeError, match="seeds must be"):
        tg.tractogram(fod, [1, 2, 3])
    with pytest.raises(TypeError, match="algorithm must be"):
        tg.tractogram(fod, 0, algorithm="transport")
    with pytest.raises(TypeError, match="domain must be"):
        tg.tractogram(fod, np.empty((0, 8), np.float32), domain="mask")
    with pytest.raises(ValueError, match="non-negative integer"):
        tg.tractogram(fod, -1)
    with pytest.raises(ValueError, match="four-dimensional"):
        tg.tractogram(tg.Nifti1Image(np.ones((2, 2, 2)), np.eye(4)), 0)


def test_tractogram_model_checks_and_empty_results():
    fod15 = tg.Nifti1Image(np.ones((2, 2, 2, 15), np.float32), np.eye(4))
    with pytest.raises(ValueError, match="only DTI and fODF"):
        tg.tractogram(fod15, 0)
    fod45 = tg.Nifti1Image(np.ones((2, 2, 2, 45), np.float32), np.eye(4))
    alg = tg.algorithm.Transport(tg.local.RealSymmetricSphericalHarmonics(15))
    with pytest.raises(ValueError, match="15 != 45"):
        tg.tractogram(fod45, 0, algorithm=alg)
    assert len(tg.tractogram(fod45, 0).streamlines) == 0
    assert len(tg.tractogram(fod45, np.empty((0, 8), np.float32)).streamlines) == 0
    # a 15-coefficient field passes when given as a field object with an algorithm
    field = tg.field.Image(fod15)
    alg15 = tg.algorithm.Transport(tg.local.RealSymmetricSphericalHarmonics(15))
    assert len(tg.tractogram(field, 0, algorithm=alg15).streamlines) == 0


def test_zero_points_budget_matches_reference_error():
    """A maximum length below save_at gives an empty point buffer (opencl.py:323-324)."""
    with pytest.raises(ValueError, match="nbytes must be positive"):
        tg.tracking._n_steps(1.0, 0.5)


def test_from_shape():
    """test/test_local.py:8-24"""
    assert isinstance(tg.local.from_shape((10, 10, 1, 6)), tg.local.DiffusionTensorImaging)
    sh = tg.local.from_shape((10, 10, 1, 45))
    assert isinstance(sh, tg.local.RealSymmetricSphericalHarmonics) and sh.n_parameters == 45
    assert sh.opencl_model == "MODEL_SYMMETRIC_REAL_SPHERICAL_HARMONICS"
    with pytest.raises(ValueError, match="only DTI and fODF"):
        tg.local.from_shape((10, 10, 1, 12))
    with pytest.raises(ValueError, match="coefficient dimension"):
        tg.local.from_shape(())


def test_unsupported_plugins_fail_loudly():
    class Custom(tg.local.BaseLocalModel):
        def evaluate(self, parameters, orientations):
            return np.zeros((len(orientations), 3))

    with pytest.raises(NotImplementedError):
        tg.local.model_id(Custom(3))
    with pytest.raises(NotImplementedError):
        tg.local.model_id(tg.local.RealSymmetricSphericalHarmonics(46))


def test_seed_validation():
    """test/test_seeds.py (validate_seed_array) and seeds.py:35-54"""
    good = np.array([[0, 0, 0, 1, 1, 0, 0, 0]], np.float64)
    out = tg.seeds.validate_seed_array(good)
    assert out.dtype == np.float32 and out.flags.c_contiguous
    with pytest.raises(ValueError, match=r"shape \(n_seeds, 8\)"):
        tg.seeds.validate_seed_array(np.zeros((2, 7)))
    with pytest.raises(ValueError, match="homogeneous"):
        tg.seeds.validate_seed_array(np.zeros((2, 8)))


def test_from_mask_and_empty_requests():
    mask = np.zeros((4, 5, 6))
    mask[1:3, 2:4, 3:5] = 1
    img = tg.Nifti1Image(mask, np.eye(4))
    np.random.seed(0)
    s = tg.seeds.from_mask(img, 500)
    assert s.shape == (500, 8)
    assert np.all(s[:, 3] == 1) and np.all(s[:, 7] == 0)
    assert np.allclose(np.linalg.norm(s[:, 4:7], axis=1), 1, atol=1e-6)
    assert np.all(tg.domain.Image(img).contains(s[:, :3]))
    assert tg.seeds.from_mask(img, 0).shape == (0, 8)
    assert tg.seeds.from_fod(tg.Nifti1Image(np.ones((2, 2, 2, 45)), np.eye(4)), 0).shape == (0, 8)


def test_from_fod_numpy_path():
    """seeds.py:218-240: NumPy path on a single-voxel x-aligned FOD."""
    d = tg.core.fibonacci_sphere(300)
    az, co, _ = tg.core.cart2sph(*d.T)
    Y, _ = tg.core.ishtmtx(az, co, 45)
    coef = np.linalg.lstsq(Y, np.exp(20 * (d[:, 0] ** 2 - 1)), rcond=None)[0]
    fod = tg.Nifti1Image(coef.reshape(1, 1, 1, 45), np.eye(4))
    np.random.seed(3)
    s = tg.seeds.from_fod(fod, 200, use_opencl=False)
    assert s.shape == (200, 8)
    assert np.mean(np.abs(s[:, 4])) > 0.8


def test_domain_and_field_constructors():
    """test/test_domain.py:26-31, 147-150; field.py:56-57"""
    with pytest.raises(ValueError, match="Only 3D images"):
        tg.domain.Image(tg.Nifti1Image(np.zeros((3, 3, 3, 3)), np.eye(4)))
    with pytest.raises(ValueError, match="at least one nonzero voxel"):
        tg.domain.Image(tg.Nifti1Image(np.zeros((2, 2, 2)), np.eye(4)))
    with pytest.raises(ValueError, match="Only 4D images"):
        tg.field.Image(tg.Nifti1Image(np.zeros((3, 3, 3)), np.eye(4)))
    d = tg.domain.Image(tg.Nifti1Image(np.ones((1, 1, 1)), np.eye(4)))
    np.testing.assert_array_equal(d.contains(np.array([[-0.5, 0, 0], [0.49, 0.49, 0.49], [0.5, 0, 0]])),
                                  [True, True, False])
    data = np.arange(64, dtype=np.float32).reshape(4, 4, 4, 1)
    f = tg.field.Image(tg.Nifti1Image(data, np.eye(4)))
    pts = np.array([[0.5, 1.5, 2.5], [1.5, 0.5, 0.5], [-0.5, 2.5, 2.5]], np.float32)
    np.testing.assert_array_equal(f.evaluate(pts), data[[0, 2, 0], [2, 0, 2], [2, 0, 2]])


def test_numpy_reference_methods():
    """test/test_algorithm.py:119-130 (exps2) and the float64 models."""
    o = np.array([[0.0, 0.0, 1.0], [1.0, 0.0, 0.0]])
    t = np.array([[0.0, 0.0, 0.0], [0.0, 0.3, 0.0]])
    r = tg.algorithm.exps2(o, t, 1.0)
    np.testing.assert_allclose(r[0], o[0])
    np.testing.assert_allclose(r[1], [np.cos(0.3), np.sin(0.3), 0.0], atol=1e-7)
    assert tg.local.DiffusionTensorImaging().evaluate(np.empty((0, 6)), np.empty((0, 3))).shape == (0, 3)
    model = tg.local.RealSymmetricSphericalHarmonics(15)
    alg = tg.algorithm.Transport(model, step_size=0.01)
    p = np.zeros((3, 15))
    p[:, 0] = 1.0
    out = alg.update_orientation(p, np.eye(3))
    np.testing.assert_allclose(out, np.eye(3), atol=1e-12)


def test_diffusion_rng_seed_sequence():
    """algorithm.py:239-241: one uint32 draw from default_rng(seed) per call."""
    a = tg.algorithm.Diffusion(tg.local.RealSymmetricSphericalHarmonics(15), seed=1234)
    rng = np.random.default_rng(1234)
    for _ in range(3):
        assert a.get_rng_seed() == int(rng.integers(0, np.iinfo(np.uint32).max, dtype=np.uint32))
    with pytest.raises(ValueError):
        tg.algorithm.Diffusion(tg.local.RealSymmetricSphericalHarmonics(15), rng="xorshift")


def test_array_sequence_and_tractogram():
    arrays = [np.arange(6, dtype=np.float32).reshape(2, 3), np.zeros((0, 3), np.float32),
              np.ones((3, 3), np.float32)]
    seq = tg.ArraySequence.from_arrays(arrays)
    assert len(seq) == 3 and [len(s) for s in seq] == [2, 0, 3]
    np.testing.assert_array_equal(seq[2], arrays[2])
    np.testing.assert_array_equal(seq[-1], arrays[2])
    sub = seq[np.array([True, False, True])]
    assert len(sub) == 2 and len(sub.get_data()) == 5
    # non-contiguous offsets (as produced by overflow waves) are allowed
    seq2 = tg.ArraySequence(np.arange(15, dtype=np.float32).reshape(5, 3), [3, 0], [2, 3])
    np.testing.assert_array_equal(seq2.get_data()[:2], np.arange(9, 15, dtype=np.float32).reshape(2, 3))
    t = tg.Tractogram(arrays, affine_to_rasmm=np.eye(4))
    assert len(t) == 3


def test_tck_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    arrays = [rng.normal(size=(n, 3)).astype(np.float32) for n in (1, 5, 0, 17)]
    t = tg.Tractogram(arrays, affine_to_rasmm=np.eye(4))
    path = tmp_path / "x.tck"
    tg.save_tck(path, t)
    raw = path.read_bytes()
    assert raw.startswith(b"mrtrix tracks\n") and b"datatype: Float32LE\n" in raw and b"count: 0000000004" in raw
    back = tg.load_tck(path)
    got = [s for s in back.streamlines]
    nonempty = [a for a in arrays if len(a)]
    assert len(got) >= len(nonempty)
    for a, b in zip(nonempty, [g for g in got if len(g)]):
        np.testing.assert_array_equal(a, b)


def test_tck_writer_streams_packed_batches(tmp_path):
    """Batches appended as packed (points, lengths, offsets) give the same bytes
    as one save_tck of the whole set, non-consecutive offsets included."""
    rng = np.random.default_rng(1)
    lengths = rng.integers(1, 30, 200)
    arrays = [rng.normal(size=(n, 3)).astype(np.float32) for n in lengths]
    whole = tmp_path / "whole.tck"
    tg.save_tck(whole, tg.Tractogram(arrays, affine_to_rasmm=np.eye(4)))
    streamed = tmp_path / "streamed.tck"
    with tg.TckWriter(streamed) as w:
        for lo in range(0, 200, 64):
            part = arrays[lo: lo + 64]
            # packed with a gap before each streamline and a fourth column, as the GPU layout has
            gap = 2
            offsets = np.cumsum([0] + [len(a) + gap for a in part])[:-1] + gap
            pts = np.full((int(offsets[-1]) + len(part[-1]) + 3, 4), 7.0, np.float32)
            for o, a in zip(offsets, part):
                pts[o: o + len(a), :3] = a
            w.append(pts, [len(a) for a in part], offsets)
        w.append(np.empty((0, 3), np.float32), [])
    assert streamed.read_bytes() == whole.read_bytes()
    back = tg.load_tck(streamed)
    assert len(back.streamlines) == 200
    for a, b in zip(arrays, back.streamlines):
        np.testing.assert_array_equal(a, b)


def test_tck_writer_applies_affine(tmp_path):
    a = np.array([[1, 2, 3], [4, 5, 6]], np.float32)
    affine = np.diag([2.0, 2.0, 2.0, 1.0])
    affine[:3, 3] = [1, 0, -1]
    path = tmp_path / "a.tck"
    tg.save_tck(path, tg.Tractogram([a], affine_to_rasmm=affine))
    back = tg.load_tck(path).streamlines[0]
    np.testing.assert_array_equal(back, a * 2 + np.array([1, 0, -1], np.float32))


def test_seed_files_round_trip(tmp_path):
    """seeds.py:243-303"""
    np.random.seed(0)
    mask = tg.Nifti1Image(np.ones((3, 3, 3)), np.eye(4))
    s = tg.seeds.from_mask(mask, 20)
    for suffix in (".txt", ".tck"):
        path = tmp_path / f"seeds{suffix}"
        tg.seeds.save(path, s)
        back = tg.seeds.load(path)
        np.testing.assert_allclose(back, s, atol=1e-5)
    with pytest.raises(ValueError, match="Unknown file type"):
        tg.seeds.save(tmp_path / "x.vtk", s)


def test_write_tractogram_without_seeds(tmp_path):
    from tractography_b200 import synthetic

    fod, mask = synthetic.config0(n=8)
    for suffix in (".tck", ".trx"):
        path = tmp_path / f"empty{suffix}"
        assert tg.write_tractogram(path, fod, np.empty((0, 8), np.float32), mask) == 0
        back = tg.load_tck(path) if suffix == ".tck" else tg.load_trx(path)[0]
        assert len(back.streamlines) == 0
    with pytest.raises(ValueError, match="Unknown tractogram file type"):
        tg.write_tractogram(tmp_path / "x.vtk", fod, np.empty((0, 8), np.float32), mask)
    with pytest.raises(ValueError, match="save_at must be finite and positive"):
        tg.write_tractogram(tmp_path / "x.tck", fod, np.empty((0, 8), np.float32), mask, save_at=0.0)
