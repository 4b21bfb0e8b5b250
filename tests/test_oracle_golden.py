"""Pins the CPU oracle against the reference's own known answers and golden tables.

Each test names the reference test (or source lines) whose assertion it restates.
"""
import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = json.loads((Path(__file__).parent / "golden" / "spectral_tables.json").read_text())


def dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def test_tables_match_reference_source(oracle_lib):
    smits = np.zeros(7 * 36)
    m = np.zeros(3 * 36)
    sun = np.zeros(36)
    oracle_lib.or_tables(dp(smits), dp(m), dp(sun))
    np.testing.assert_array_equal(smits.reshape(7, 36), np.array(GOLDEN["smits_basis"]))
    np.testing.assert_array_equal(m.reshape(3, 36), np.array(GOLDEN["spectrum_to_rgb"]))
    np.testing.assert_array_equal(sun, np.array(GOLDEN["sun_spectrum"]))


def test_host_tables_match_reference_source():
    from naivetrace_b200 import spectral
    s, m, sun = spectral.tables()
    np.testing.assert_array_equal(s, np.array(GOLDEN["smits_basis"]))
    np.testing.assert_array_equal(m, np.array(GOLDEN["spectrum_to_rgb"]))
    np.testing.assert_array_equal(sun, np.array(GOLDEN["sun_spectrum"]))
    np.testing.assert_array_equal(spectral.WAVELENGTHS, np.array(GOLDEN["wavelengths"]))


def test_rgb_conversion_round_trip(oracle_lib):
    """TEST(Spectral, RGBConversion), tests.cxx:255-286."""
    tol = GOLDEN["rgb_round_trip_tolerance"]
    for trial in GOLDEN["rgb_round_trip_trials"]:
        rgb = np.array(trial, dtype=np.float64)
        spec = np.zeros(36)
        oracle_lib.or_rgb_to_spectrum(dp(rgb), dp(spec))
        assert spec.min() >= -1e-12 and spec.max() <= 1.01
        back = np.zeros(3)
        oracle_lib.or_spectrum_to_rgb(dp(spec), dp(back))
        np.testing.assert_allclose(back, rgb, atol=tol)


def test_rgb_conversion_linearity(oracle_lib):
    """TEST(Spectral, RGBConversionLinearity), tests.cxx:289-307."""
    specs = [np.zeros(36) for _ in range(3)]
    specs[0][0] = 1
    specs[1][2] = 1
    specs[2][35] = 1

    def to_rgb(s):
        out = np.zeros(3)
        s = np.ascontiguousarray(s)
        oracle_lib.or_spectrum_to_rgb(dp(s), dp(out))
        return out

    for a, b in [(0, 1), (0, 2), (1, 2)]:
        d = to_rgb(specs[a] + specs[b]) - to_rgb(specs[a]) - to_rgb(specs[b])
        assert np.abs(d).max() <= 1e-3


def test_rgb_selection_round_trip(oracle_lib):
    """TEST(Spectral, RGBConversionSelection), tests.cxx:310-327."""
    rgb = np.array([0.8, 0.2, 0.6])
    acc = np.zeros(3)
    for lam in range(0, 34, 3):
        idx = np.array([lam, lam + 1, lam + 2], np.int32)
        sel = np.zeros(3)
        oracle_lib.or_rgb_to_selection(dp(rgb), ip(idx), dp(sel))
        out = np.zeros(3)
        oracle_lib.or_selection_to_rgb(dp(sel), ip(idx), dp(out))
        acc += out
    np.testing.assert_allclose(acc, rgb, atol=1e-2)


def _n(v):
    v = np.asarray(v, dtype=np.float64)
    return v / np.linalg.norm(v)


def test_reflected(oracle_lib):
    """TEST(TestMath, Reflected), tests.cxx:121-132."""
    w_in = _n([0, 1, 2])
    exp = _n([0, 1, -2])
    for n in ([0, 1, 0], [0, -1, 0]):
        out = np.zeros(3)
        oracle_lib.or_reflected(dp(w_in), dp(np.array(n, float)), dp(out))
        assert out @ exp >= 0.99


def test_refracted(oracle_lib):
    """TEST(TestMath, Refracted), tests.cxx:135-161."""
    n = np.array([0.0, 1.0, 0.0])
    w1 = _n([0, 1, 2])
    w2 = np.zeros(3)
    assert oracle_lib.or_refracted(dp(w1), dp(n), 1.0 / 1.1, dp(w2)) == 1
    w3 = np.zeros(3)
    assert oracle_lib.or_refracted(dp(w2), dp(n), 1.1 / 1.0, dp(w3)) == 1
    np.testing.assert_allclose(w3, w1, atol=1e-3)
    nflip = np.array([0.0, -1.0, 0.0])
    w4 = np.zeros(3)
    assert oracle_lib.or_refracted(dp(w1), dp(nflip), 1.0 / 1.1, dp(w4)) == 1
    np.testing.assert_allclose(w4, w2, atol=1e-3)
    w5 = _n([0, 1, 100])
    assert oracle_lib.or_refracted(dp(w5), dp(nflip), 1.2, dp(np.zeros(3))) == 0


def test_refracted_half_vector(oracle_lib):
    """TEST(TestMath, RefractedHalfVector[Degenerate]), tests.cxx:164-189."""
    for w1, w2 in ((_n([0, 3, 1]), _n([0, -1, 0])), (np.array([0, 1.0, 0]), np.array([0, -1.0, 0]))):
        h = np.zeros(3)
        assert oracle_lib.or_half_vector_refracted(dp(w1), dp(w2), 1.0 / 1.5, dp(h)) == 1
        wr = np.zeros(3)
        assert oracle_lib.or_refracted(dp(w1), dp(h), 1.0 / 1.5, dp(wr)) == 1
        assert abs(wr[0] - w2[0]) < 1e-3


def test_half_vector(oracle_lib):
    """TEST(TestMath, HalfVector[Degenerate]), tests.cxx:192-212."""
    for w1, w2 in ((_n([0, 3, 1]), _n([0, -1, 0])), (np.array([0, 1.0, 0]), np.array([0, -1.0, 0]))):
        h = np.zeros(3)
        oracle_lib.or_half_vector(dp(w1), dp(w2), dp(h))
        wr = np.zeros(3)
        oracle_lib.or_reflected(dp(w1), dp(h), dp(wr))
        assert abs(wr[0] - w2[0]) < 1e-3


def test_fresnel_limits(oracle_lib):
    # Normal incidence on glass: ((1 - 1.5) / (1 + 1.5))^2 = 0.04.
    assert abs(oracle_lib.or_fresnel(1.0, 1.0 / 1.5) - 0.04) < 1e-12
    # Total internal reflection from inside.
    assert oracle_lib.or_fresnel(0.1, 1.5) == 1.0


def test_pcg32_known_answer(oracle_lib):
    """PCG32 reference output for srandom(42, 54) (O'Neill's pcg32 demo), which pins the
    generator the reference seeds through pcg32::seed (sampler.cxx:366-368)."""
    out = np.zeros(6, np.uint32)
    oracle_lib.or_pcg32_stream(42, 54, 6, out.ctypes.data_as(C.POINTER(C.c_uint32)))
    assert [hex(int(x)) for x in out] == ["0xa15c02b7", "0x7b47f409", "0xba1d3330", "0x83d2f293", "0xbfa4784b",
                                          "0xcbed606e"]


def test_uniform_int_range_and_balance(oracle_lib):
    """RandGen::UniformInt (sampler.cxx:384-391): inclusive range, unbiased."""
    out = np.zeros(120000, np.int32)
    oracle_lib.or_uniform_int_stream(7, 3, 0, 11, len(out), ip(out))
    assert out.min() == 0 and out.max() == 11
    counts = np.bincount(out, minlength=12)
    expected = len(out) / 12
    assert np.all(np.abs(counts - expected) < 5 * np.sqrt(expected))
