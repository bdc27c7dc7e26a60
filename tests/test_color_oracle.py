"""The oracle's colour and metric restatements against the reference's own known answers:
crates/mars-core/tests/known_answers.rs (mse / psnr) and metrics.rs's ycbcr tests."""
import math

import numpy as np

import mars_b200 as mb
from oracle import oracle as orc


def test_mse_psnr_known_answers():
    # known_answers.rs:49-76
    a = np.array([[10, 20], [30, 40]], np.uint8)
    b = np.array([[11, 18], [33, 36]], np.uint8)
    assert orc.mse(a, b) == 7.5
    a = np.full((4, 4), 100, np.uint8)
    b = np.full((4, 4), 101, np.uint8)
    assert orc.mse(a, b) == 1.0
    assert abs(mb.psnr_from_mse(orc.mse(a, b)) - 48.130_803_608_679_02) < 1e-11
    assert mb.psnr_from_mse(0.0) is None
    z, f = np.zeros((8, 8), np.uint8), np.full((8, 8), 255, np.uint8)
    assert orc.mse(z, f) == 65025.0 and abs(mb.psnr_from_mse(65025.0)) < 1e-12
    big = np.full((1024, 1024), 255, np.uint8)
    assert orc.mse(np.zeros_like(big), big) == 65025.0


def test_ycbcr_gray_round_trip_is_exact():
    # metrics.rs ycbcr_roundtrip_is_exact_for_gray_input
    v = np.array([0, 1, 128, 255], np.uint8)
    y, cb, cr = orc.ycbcr(v, v, v)
    assert cb.tolist() == [128] * 4 and cr.tolist() == [128] * 4
    r, g, b = orc.rgb_from_ycbcr(y, cb, cr)
    assert r.tolist() == v.tolist() and g.tolist() == v.tolist() and b.tolist() == v.tolist()


def test_ycbcr_round_trip_within_two_lsb():
    # metrics.rs ycbcr_roundtrip_is_nearly_lossless
    n = 64
    yy, xx = np.mgrid[0:n, 0:n]
    r = ((xx * 4) % 256).astype(np.uint8)
    g = ((yy * 4) % 256).astype(np.uint8)
    b = (((xx + yy) * 3) % 256).astype(np.uint8)
    back = orc.rgb_from_ycbcr(*orc.ycbcr(r, g, b))
    for o, d in zip((r, g, b), back):
        assert np.abs(o.astype(int) - d.astype(int)).max() <= 2


def test_downsample_upsample():
    p = np.arange(35, dtype=np.uint8).reshape(5, 7)
    d = orc.downsample_box(p)
    assert d.shape == (3, 4)
    # corner block (sum + 2) / 4, and the replicated last column / row
    assert d[0, 0] == (0 + 1 + 7 + 8 + 2) // 4
    assert d[0, 3] == (6 + 6 + 13 + 13 + 2) // 4
    assert d[2, 3] == (34 * 4 + 2) // 4
    u = orc.upsample_nearest(d, 7, 5)
    assert u.shape == (5, 7) and u[4, 6] == d[2, 3] and u[1, 1] == d[0, 0]
    assert math.isclose(orc.mse(u, u), 0.0)
