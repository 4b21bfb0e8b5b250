"""The quasi-random sampler of the null-path tracer (QuasiRandomSequence, sampler.cxx:254-331)
in the CPU oracle, pinned against independent and published values.

1. Generator matrices: dimensions 0-2 give the standard Sobol points (an independent
   implementation, scipy's unscrambled Sobol sequence, in Gray-code order); dimensions
   3-10 agree with it on their first 2^s points (the initial direction numbers, shared by
   both Joe-Kuo tables) and then differ, because the reference's generator pairs the
   polynomial's coefficients with the direction numbers in the opposite order; that
   recurrence is pinned by the worked example of the reference's generator notebook
   (misc/SobolSequenceGeneratorMatrices.ipynb: s = 3, a = 2, m = 1, 3, 7 gives m_4 = 5,
   m_5 = 7).
2. Every one of the 4096 dimensions is a (0, 1)-sequence: its first 2^m points fall one in
   each interval of length 2^-m.
3. The rotation table equals the reference's first and last entries
   (sampler_tables.cxx:4, :130).
4. Draw order: the k-th Uniform01 of subsequence id is dimension (id << 6) + 2 + k plus
   the pixel's x rotation modulo 1, the 63rd and later come from PCG32, UniformUnitSquare
   is dimensions (id << 6) and (id << 6) + 1 with the (x, y) rotation, and setting the
   subsequence restarts the count.
"""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from oracle.oracle import load

DATA = Path(__file__).resolve().parents[1] / "naivetrace_b200" / "csrc" / "tt_sobol_data.h"


def _u32p(a):
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def sobol(dim, points):
    lib = load()
    pts = np.ascontiguousarray(points, dtype=np.uint32)
    out = np.zeros(len(pts))
    assert lib.or_sobol(dim, len(pts), _u32p(pts), _dp(out)) == 0
    return out


def _table():
    txt = DATA.read_text()
    a = txt.index("tt_sobol_sam[] = {")
    sam = [int(v) for v in re.findall(r"\d+", txt[a + 18:txt.index("};", a)])]
    b = txt.index("tt_rotation_offsets[] = {")
    rot = [float(v) for v in re.findall(r"([-0-9.eE]+)f", txt[b:txt.index("};", b)])]
    return sam, np.array(rot, np.float32).reshape(-1, 2)


def test_dims_0_to_2_are_the_standard_sobol_sequence():
    qmc = pytest.importorskip("scipy.stats.qmc")
    n = 4096
    k = np.arange(n, dtype=np.uint32)
    ref = qmc.Sobol(d=11, scramble=False).random(n)
    gray = k ^ (k >> 1)
    for dim in range(3):
        np.testing.assert_array_equal(sobol(dim, gray), ref[:, dim])
    # Dimensions 3-10: the same first 2^s points, then the reference's recurrence.
    sam, _ = _table()
    pos = 0
    for dim in range(1, 11):
        s = sam[pos]
        pos += 2 + s
        if dim < 3:
            continue
        got = sobol(dim, gray[: 1 << s])
        np.testing.assert_array_equal(got, ref[: 1 << s, dim])
        assert not np.array_equal(sobol(dim, gray), ref[:, dim])


def test_generator_recurrence_worked_example():
    lib = load()
    m = np.array([1, 3, 7], np.uint16)
    out = np.zeros(32, np.uint32)
    lib.or_sobol_matrix(3, 2, m.ctypes.data_as(C.POINTER(C.c_uint16)), _u32p(out))
    direction = [int(out[k]) >> (31 - k) for k in range(6)]
    assert direction[:5] == [1, 3, 7, 5, 7], direction


def test_every_dimension_is_stratified():
    n = 1024
    k = np.arange(n, dtype=np.uint32)
    for dim in range(4096):
        x = sobol(dim, k)
        cells = np.floor(x * n).astype(int)
        assert np.array_equal(np.sort(cells), np.arange(n)), dim


def test_tables():
    sam, rot = _table()
    assert rot.shape == (128 * 128, 2)
    assert np.all((rot >= 0) & (rot < 1))
    np.testing.assert_array_equal(rot[0], np.array([0.24019504, 0.13671502], np.float32))
    np.testing.assert_array_equal(rot[1], np.array([0.14869094, 0.6305471], np.float32))
    np.testing.assert_array_equal(rot[-1], np.array([0.7793244, 0.6110513], np.float32))
    # 4095 dimensions of (s, a, m_1..m_s) with odd m_i < 2^i.
    pos, dims = 0, 0
    while pos < len(sam):
        s, a = sam[pos], sam[pos + 1]
        m = sam[pos + 2: pos + 2 + s]
        assert len(m) == s and a < (1 << max(s - 1, 0)) + 1
        assert all(v % 2 == 1 and v < (1 << (i + 1)) for i, v in enumerate(m))
        pos += 2 + s
        dims += 1
    assert dims == 4095


def test_draw_order():
    lib = load()
    _, rot = _table()
    px, py, point = 130, 5, 37
    r = rot[(px % 128) + (py % 128) * 128].astype(np.float64)
    ops = [2 + 5] + [0] * 64 + [1] + [2 + 9, 0, 1]
    ops_a = np.array(ops, np.int32)
    out = np.zeros(64 + 2 + 1 + 2)
    assert lib.or_qmc_draws(px, py, point, len(ops), ops_a.ctypes.data_as(C.POINTER(C.c_int32)), 3, _dp(out)) == 0
    wrap = lambda x: x - 1.0 if x >= 1.0 else x
    for k in range(62):
        assert out[k] == wrap(sobol(5 * 64 + 2 + k, [point])[0] + r[0])
    # Draws 63 and 64 come from PCG32: in [0, 1), not the Sobol dimensions.
    assert all(0 <= out[k] < 1 for k in (62, 63))
    assert out[64] == wrap(sobol(5 * 64, [point])[0] + r[0])
    assert out[65] == wrap(sobol(5 * 64 + 1, [point])[0] + r[1])
    assert out[66] == wrap(sobol(9 * 64 + 2, [point])[0] + r[0])
    assert out[67] == wrap(sobol(9 * 64, [point])[0] + r[0])


def test_pt2_qmc_converges_faster_to_the_same_image():
    """pt2 with quasi-random points renders the same image as with PCG32 (1024 spp means
    within 3 %) and with lower relMSE at 64 spp (direct lighting of the Cornell box)."""
    from naivetrace_b200 import abi, scenes
    from naivetrace_b200.scene import make_params
    from oracle.oracle import OracleScene, combine

    scene = scenes.cornell_box(16, 16)

    def img(p, spp, seed):
        o = OracleScene(scene, p)
        acc, light, splat = o.render(spp, seed=seed)
        return combine(acc, light, spp, splat, o.npix).reshape(-1, 3)

    pp = make_params(max_ray_depth=3, algo=abi.ALGO_PT2)
    pq = make_params(max_ray_depth=3, algo=abi.ALGO_PT2, qmc=True)
    R = np.mean([img(pp, 1024, 1000 + k) for k in range(4)], axis=0)
    np.testing.assert_allclose(img(pq, 1024, 5).mean(0), R.mean(0), rtol=0.03)
    e_p = np.mean([np.mean((img(pp, 64, 10 + k) - R) ** 2 / (R * R + 1e-2)) for k in range(4)])
    e_q = np.mean([np.mean((img(pq, 64, 10 + k) - R) ** 2 / (R * R + 1e-2)) for k in range(4)])
    assert e_q < 0.85 * e_p, (e_p, e_q)
