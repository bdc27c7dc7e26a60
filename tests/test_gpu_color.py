"""The colour input and metric kernels (color.cu) against the oracle, bit-exact, and the
colour encode/decode pipeline (color.rs:400-528 without regions) end to end."""
import numpy as np
import pytest

import mars_b200 as mb
from mars_b200 import color, synthetic
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = mb.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("shape", [(64, 64), (37, 53), (1, 7), (3, 2), (256, 384)])
def test_ycbcr_both_ways(ctx, shape):
    rng = np.random.default_rng(sum(shape))
    r, g, b = (rng.integers(0, 256, shape, dtype=np.uint8) for _ in range(3))
    got = ctx.ycbcr(r, g, b)
    want = orc.ycbcr(r, g, b)
    for x, y in zip(got, want):
        assert np.array_equal(x, y)
    back = ctx.rgb_from_ycbcr(*got)
    for x, y in zip(back, orc.rgb_from_ycbcr(*want)):
        assert np.array_equal(x, y)


def test_every_rgb_value_on_one_axis(ctx):
    # All 2^24 colours would be 48 MB per plane; every (r, g, b) with r, g, b in 0..255 in
    # steps covers the rounding boundaries of each coefficient.
    v = np.arange(256, dtype=np.uint8)
    r, g, b = np.meshgrid(v, v[::3], v[::5], indexing="ij")
    got = ctx.ycbcr(r, g, b)
    for x, y in zip(got, orc.ycbcr(r, g, b)):
        assert np.array_equal(x, y)
    for x, y in zip(ctx.rgb_from_ycbcr(r, g, b), orc.rgb_from_ycbcr(r, g, b)):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("shape", [(64, 64), (37, 53), (1, 1), (1, 9), (513, 257)])
def test_downsample_and_upsample(ctx, shape):
    rng = np.random.default_rng(shape[0] * 7 + shape[1])
    p = rng.integers(0, 256, shape, dtype=np.uint8)
    d = ctx.downsample_box(p)
    assert np.array_equal(d, orc.downsample_box(p))
    h, w = shape
    assert np.array_equal(ctx.upsample_nearest(d, w, h), orc.upsample_nearest(d, w, h))


@pytest.mark.parametrize("n", [1, 15, 16, 17, 4096, 1 << 20, (1 << 20) + 3])
def test_mse(ctx, n):
    rng = np.random.default_rng(n)
    a = rng.integers(0, 256, (1, n), dtype=np.uint8)
    b = rng.integers(0, 256, (1, n), dtype=np.uint8)
    assert ctx.mse(a, b) == orc.mse(a, b)
    assert ctx.mse(a, a) == 0.0
    assert ctx.mse(np.zeros((1, n), np.uint8), np.full((1, n), 255, np.uint8)) == 65025.0


def test_color_pipeline_matches_the_oracle_pipeline(ctx):
    # Config 3 in miniature: RGB -> Y + 4:2:0 Cb/Cr -> per-plane encodes -> MARC container,
    # then decode back; the oracle path runs the same steps with its own restatements.
    rgb = synthetic.rgb(96, 64, 2)
    y_p = dict(min_size=4, max_size=16, shift=2, lam=200.0)
    c_p = dict(min_size=4, max_size=16, shift=2, lam=400.0)
    params = color.ColorEncodeParams(mb.make_params(**y_p), mb.make_params(**c_p))
    data, stats = color.encode_color(ctx, rgb, params)

    y, cb, cr = orc.ycbcr(rgb[..., 0], rgb[..., 1], rgb[..., 2])
    streams = []
    for plane, kw in ((y, y_p), (orc.downsample_box(cb), c_p), (orc.downsample_box(cr), c_p)):
        h, l, res, _, _ = orc.encode(plane, orc.make_params(**kw), allowed_modes=(1, 1, 1, 1))
        streams.append(mb.format_write(mb.Header(*[getattr(h, f) for f, _ in h._fields_]), l, res))
    assert data == color.write_container(color.MODE_RGB_420, streams)
    assert stats.cb_bytes == len(streams[1])

    out = color.decode_color(ctx, data, 10)
    assert out.shape == rgb.shape
    planes = []
    for s in streams:
        h, l, res = mb.format_read(s)
        planes.append(orc.decode(orc.Header(*[getattr(h, f) for f, _ in h._fields_]), l, 10, res))
    H, W = planes[0].shape
    ref = orc.rgb_from_ycbcr(planes[0], orc.upsample_nearest(planes[1], W, H),
                             orc.upsample_nearest(planes[2], W, H))
    assert np.array_equal(out, np.stack(ref, axis=-1))
    assert mb.psnr_from_mse(ctx.mse(out[..., 1], rgb[..., 1])) > 15.0


def test_zoomed_and_auto_colour_decodes(ctx):
    rgb = synthetic.rgb(96, 64, 5)
    kw = dict(min_size=4, max_size=16, shift=2, lam=200.0)
    params = color.ColorEncodeParams(mb.make_params(**kw), mb.make_params(**kw))
    data, _ = color.encode_color(ctx, rgb, params)
    mode, streams = color.read_container(data)
    oplanes = []
    for s in streams:
        h, l, res = mb.format_read(s)
        oh = orc.Header(*[getattr(h, f) for f, _ in h._fields_])
        zh, zl = orc.zoom_leaves(oh, l, 2.0)
        oplanes.append(orc.decode(zh, zl, 10))
    H, W = oplanes[0].shape
    ref = np.stack(orc.rgb_from_ycbcr(oplanes[0], orc.upsample_nearest(oplanes[1], W, H),
                                      orc.upsample_nearest(oplanes[2], W, H)), axis=-1)
    assert np.array_equal(color.decode_color_zoomed(ctx, data, 10, 2.0), ref)
    out, used = color.decode_color_auto(ctx, data, 1, 40)
    uses = []
    oplanes = []
    for s in streams:
        h, l, res = mb.format_read(s)
        oh = orc.Header(*[getattr(h, f) for f, _ in h._fields_])
        p, n = orc.decode_until_stable(oh, l, 1, 40, res)
        oplanes.append(p)
        uses.append(n)
    H, W = oplanes[0].shape
    ref = np.stack(orc.rgb_from_ycbcr(oplanes[0], orc.upsample_nearest(oplanes[1], W, H),
                                      orc.upsample_nearest(oplanes[2], W, H)), axis=-1)
    assert used == max(uses) and np.array_equal(out, ref)
