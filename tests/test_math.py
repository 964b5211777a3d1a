"""Accuracy of the shared binary32 math layer and of the SH basis (CPU, through the oracle).

The math layer (csrc/tg_fmath.h) must stay within 2 ulp of double-precision
libm; the oracle's table-driven SH evaluation must match the float64 SciPy
basis (core.ishtmtx, the reference's core.py:36-69 convention) to float32
rounding.
"""

import numpy as np
import pytest

import tractography_b200 as tg


def ulp_error(got, want):
    got = np.asarray(got, dtype=np.float64)
    want32 = np.asarray(want, dtype=np.float32)
    spacing = np.abs(np.spacing(want32)).astype(np.float64)
    spacing[spacing == 0] = np.finfo(np.float32).smallest_subnormal
    return np.abs(got - np.asarray(want, dtype=np.float64)) / spacing


@pytest.mark.parametrize("fn", ["sin", "cos"])
def test_sincos_within_two_ulp(oracle, fn):
    x = np.linspace(-100.0, 100.0, 2_000_001, dtype=np.float32)
    got = oracle.math(fn, x)
    want = getattr(np, fn)(x.astype(np.float64))
    err = ulp_error(got, want)
    assert err.max() <= 2.0, (fn, float(err.max()), x[np.argmax(err)])


def test_exp_within_two_ulp(oracle):
    x = np.linspace(-103.0, 88.7, 2_000_001, dtype=np.float32)
    err = ulp_error(oracle.math("exp", x), np.exp(x.astype(np.float64)))
    assert err.max() <= 2.0
    special = oracle.math("exp", np.array([0.0, -200.0, 200.0, np.nan], np.float32))
    assert special[0] == 1.0 and special[1] == 0.0 and np.isinf(special[2]) and np.isnan(special[3])


def test_log_of_positive_normal_arguments_within_one_ulp(oracle):
    """The step's logarithm (Box-Muller's uniform in [2^-24, 1), 1 + e^{kx} up to 1 + e^30):
    the reduced argument's polynomial (gen_fmath_coefficients.py) stays within one ulp."""
    rng = np.random.default_rng(1)
    x = np.concatenate([
        np.arange(1, 1 << 24, 7, dtype=np.float64).astype(np.float32) * np.float32(2.0 ** -24),
        np.linspace(0.70710677, 1.0, 1_000_001, dtype=np.float32),
        np.linspace(1.0, 2.0, 1_000_001, dtype=np.float32),
        (2.0 ** rng.uniform(-125, 60, 1_000_000)).astype(np.float32),
        np.array([np.float32(2.0 ** -24), np.nextafter(np.float32(1.0), np.float32(0.0)), 1.0,
                  np.float32(0.70710677), np.float32(1.4142135)], np.float32),
    ])
    err = ulp_error(oracle.math("log_pos", x), np.log(x.astype(np.float64)))
    assert err.max() <= 1.0, (float(err.max()), x[np.argmax(err)])
    assert oracle.math("log_pos", np.array([1.0], np.float32))[0] == 0.0


def test_exps2_factors_within_two_ulp(oracle):
    """cos(n) and sin(n)/n from n2 = n^2 (the exponential map, core.cl:101-109): the
    series below n2 = 1 and the general path above agree with float64 to 2 ulp."""
    series = np.concatenate([np.linspace(1e-12, 1.0, 1_000_001, dtype=np.float32)[:-1],
                             np.array([np.nextafter(np.float32(1.0), np.float32(0.0))], np.float32)])
    n = np.sqrt(series.astype(np.float64))
    assert ulp_error(oracle.math("exps2_cos", series), np.cos(n)).max() <= 2.0
    assert ulp_error(oracle.math("exps2_sinc", series), np.sin(n) / n).max() <= 2.0
    # above n2 = 1: sin and cos of n = sqrt(n2) rounded to binary32
    general = np.linspace(1.0, 400.0, 400_001, dtype=np.float32)
    n32 = np.sqrt(general).astype(np.float64)
    assert ulp_error(oracle.math("exps2_cos", general), np.cos(n32)).max() <= 2.0
    assert ulp_error(oracle.math("exps2_sinc", general), np.sin(n32) / n32).max() <= 3.0


def test_softplus_and_slope(oracle):
    """softplus(x) = log(1 + e^{100x})/100 below 100x = 30, else x; slope 1/(1 + e^{-100x})
    (core.cl:111-120), both from one exponential."""
    x = np.linspace(-1.2, 0.6, 1_000_001, dtype=np.float32)
    x64 = x.astype(np.float64)
    want = np.where(100 * x64 < 30, np.log1p(np.exp(100 * x64)) / 100, x64)
    got = oracle.math("softplus", x).astype(np.float64)
    # log(1 + E) inherits the rounding of the binary32 sum 1 + E (half an ulp
    # of 1, divided by 100), as the reference's formula does; beyond that 3 ulp
    allowed = 3 * np.spacing(want.astype(np.float32)).astype(np.float64) + 2.0 ** -24 / 100 * 1.01
    assert np.all(np.abs(got - want) <= allowed)
    slope = oracle.math("softplus_slope", x)
    want_slope = 1 / (1 + np.exp(-100 * x64))
    assert np.abs(slope - want_slope).max() <= 4 * np.spacing(np.float32(1.0))
    assert np.all(slope[100 * x >= 30] == 1.0)
    assert np.isnan(oracle.math("softplus_slope", np.array([np.nan], np.float32))[0])
    # the drift's divisor 1 / max(softplus, 1e-6) shares the slope's division
    inv = oracle.math("softplus_inv_floor", x).astype(np.float64)
    want_inv = 1 / np.maximum(got, 1e-6)
    assert np.all(np.abs(inv - want_inv) <= 3 * np.spacing(want_inv.astype(np.float32)))


def test_cos2pi_of_24_bit_draws(oracle):
    """cos(2 pi k 2^-24) with exact integer quarter turns (Box-Muller's angle,
    core.cl:240-245): within 2 ulp of float64, or 2^-24 absolute near its zeros."""
    k = np.concatenate([np.arange(0, 1 << 24, 37, dtype=np.int64),
                        np.array([0, 1, (1 << 21) - 1, 1 << 21, (1 << 22), (1 << 24) - 1], np.int64)])
    got = oracle.math("cos2pi_u24", k.astype(np.float32)).astype(np.float64)
    want = np.cos(2 * np.pi * k.astype(np.float64) / 2.0 ** 24)
    err = np.abs(got - want)
    assert np.all(err <= np.maximum(2 * np.spacing(np.abs(want).astype(np.float32)), 2.0 ** -24))


def test_exp_up_to_30_within_two_ulp(oracle):
    """softplus's exponential (argument capped at 30): 2 ulp down to -87.3, then 0."""
    x = np.linspace(-87.3, 30.0, 2_000_001, dtype=np.float32)
    err = ulp_error(oracle.math("exp_upto30", x), np.exp(x.astype(np.float64)))
    assert err.max() <= 2.0
    below = oracle.math("exp_upto30", np.array([-87.34, -100.0, -np.inf], np.float32))
    assert np.all(below == 0.0)


def test_log_within_two_ulp(oracle):
    rng = np.random.default_rng(0)
    x = np.concatenate([
        np.linspace(0.5, 2.0, 1_000_001, dtype=np.float32),
        (2.0 ** rng.uniform(-140, 127, 1_000_000)).astype(np.float32),
    ])
    x = x[x > 0]
    err = ulp_error(oracle.math("log", x), np.log(x.astype(np.float64)))
    assert err.max() <= 2.0
    special = oracle.math("log", np.array([1.0, 0.0, -1.0, np.inf], np.float32))
    assert special[0] == 0.0 and special[1] == -np.inf and np.isnan(special[2]) and special[3] == np.inf


@pytest.mark.parametrize("C", [1, 6, 15, 28, 45])
def test_oracle_sh_basis_matches_scipy(oracle, C):
    rng = np.random.default_rng(C)
    n = 4000
    phi = rng.uniform(0, 2 * np.pi, n)
    theta = np.arccos(rng.uniform(-1, 1, n))
    o = np.stack(tg.core.sph2cart(phi, theta, 1.0), -1).astype(np.float32)
    params = (rng.normal(size=(n, C)) * 0.1).astype(np.float32)
    params[:, 0] = 40.0                     # softplus is the identity above 0.3
    got = oracle.local_evaluate(oracle.MODEL_SH, params, o)
    want = tg.local.RealSymmetricSphericalHarmonics(C).evaluate(params.astype(np.float64), o.astype(np.float64))
    scale = np.abs(want).max(axis=0)
    assert np.all(np.abs(got - want).max(axis=0) <= 5e-6 * scale + 1e-6)


def test_oracle_dti_matches_float64(oracle):
    rng = np.random.default_rng(1)
    p = rng.normal(size=(500, 6)).astype(np.float32)
    o = rng.normal(size=(500, 3)).astype(np.float32)
    o /= np.linalg.norm(o, axis=1, keepdims=True)
    got = oracle.local_evaluate(oracle.MODEL_DTI, p, o)
    want = tg.local.DiffusionTensorImaging().evaluate(p.astype(np.float64), o.astype(np.float64))
    np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-5)


def test_philox_known_answer(oracle):
    # Random123 known-answer vectors for philox4x32-10 (Salmon et al. 2011)
    assert list(oracle.philox([0, 0, 0, 0], [0, 0])) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert list(oracle.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2)) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6,
                                                                      0x6D5451FD]


def test_polynomial_coefficients_match_their_generator():
    """The fitted polynomials of tg_fmath.h are the ones gen_fmath_coefficients.py fits."""
    import importlib.util
    import re
    from pathlib import Path

    csrc = Path(__file__).resolve().parents[1] / "tractography_b200" / "csrc"
    spec = importlib.util.spec_from_file_location("gen_fmath_coefficients", csrc / "gen_fmath_coefficients.py")
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    text = (csrc / "tg_fmath.h").read_text()
    tagged = {}
    for value, tag, k in re.findall(r"(-?0x[0-9a-f.]+p-?\d+|-0\.5)f[);]*\s*/\* ([QSCPK])(\d) \*/", text):
        tagged.setdefault(tag, {})[int(k)] = float.fromhex(value) if value.startswith(("0x", "-0x")) else float(value)
    for tag, name in (("Q", "log"), ("S", "sin"), ("C", "cos"), ("P", "expc"), ("K", "expk")):
        q, _ = gen.fit(name)
        assert sorted(tagged[tag]) == list(range(len(q))), tag
        assert all(np.float32(tagged[tag][k]) == q[k] for k in range(len(q))), tag


def test_reciprocal_square_root_within_two_ulp(oracle):
    """The orientation frame's 1/rho: Lomont's estimate and three Newton steps."""
    rng = np.random.default_rng(3)
    x = np.concatenate([np.linspace(0.25, 4.0, 2_000_001, dtype=np.float32),
                        (2.0 ** rng.uniform(-100, 60, 1_000_000)).astype(np.float32),
                        np.array([2.0 ** -100, 1.0, 2.0, np.nextafter(np.float32(1.0), np.float32(0.0))],
                                 np.float32)])
    err = ulp_error(oracle.math("rsqrt_pos", x), 1.0 / np.sqrt(x.astype(np.float64)))
    assert err.max() <= 2.0, (float(err.max()), x[np.argmax(err)])
