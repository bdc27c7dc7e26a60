"""Tiny and odd geometries (crates/mars-codec/tests/tiny_geometry.rs): 1x1 .. 8x8 planes
through the encoder, the .mars container and the decoder, GPU against the oracle; and the
reference's known answer for a zero-alpha mode-3 leaf, whose residual is added in
domain-local orientation without any domain read (tiny_geometry.rs:163-219)."""
import numpy as np
import pytest

import mars_b200 as mb
from oracle import oracle as orc

SIZES = [(1, 1), (1, 5), (5, 1), (3, 5), (4, 4), (8, 8)]


def xorshift_plane(w, h):
    """The reference's image(): xorshift32 from 0x5eed1979, low byte per pixel."""
    state = 0x5EED1979
    out = np.zeros(w * h, np.uint8)
    for i in range(w * h):
        state ^= (state << 13) & 0xFFFFFFFF
        state ^= state >> 17
        state ^= (state << 5) & 0xFFFFFFFF
        out[i] = state & 0xFF
    return out.reshape(h, w)


def zero_alpha_case():
    levels = np.array([1, 2, -3, 4], np.int32)
    spatial = orc.inverse_dct2d((levels * 8.0).reshape(2, 2)).ravel()
    pixels = [int(0.5 + 64.0 / 127.0 * 255.0 + r) for r in spatial]
    orders = [[0, 1, 2, 3], [1, 3, 0, 2], [2, 0, 3, 1], [3, 2, 1, 0],
              [1, 0, 3, 2], [2, 3, 0, 1], [0, 2, 1, 3], [3, 1, 2, 0]]
    return levels, pixels, orders


def test_zero_alpha_residual_known_answer_oracle():
    levels, pixels, orders = zero_alpha_case()
    hdr = orc.Header(4, 7, 2, 2, 4, 2, 2, 32)
    for iso, order in enumerate(orders):
        leaf = np.array([(0, 0, 2, 3, 0, 64, iso, 0, 0, 0, 0)], dtype=orc.LEAF_DTYPE)
        got = orc.decode(hdr, leaf, 1, levels).ravel()
        assert list(got) == [pixels[i] for i in order], iso


@pytest.mark.gpu
def test_zero_alpha_residual_known_answer_gpu():
    levels, pixels, orders = zero_alpha_case()
    hdr = mb.Header(4, 7, 2, 2, 4, 2, 2, 32)
    with mb.Context(0) as ctx:
        for iso, order in enumerate(orders):
            leaf = np.array([(0, 0, 2, 3, 0, 64, iso, 0, 0, 0, 0)], dtype=mb.LEAF_DTYPE)
            for iters in (1, 3):
                got = ctx.decode(hdr, leaf, iters, levels).ravel()
                assert list(got) == [pixels[i] for i in order], iso


@pytest.mark.gpu
@pytest.mark.parametrize("w,h", SIZES)
@pytest.mark.parametrize("lam", [None, 2.0])
def test_tiny_planes_round_trip(w, h, lam):
    img = xorshift_plane(w, h)
    kw = dict(min_size=4, max_size=4, shift=4, lam=lam)
    with mb.Context(0) as ctx:
        for modes in ((1, 0, 1, 0), (1, 1, 1, 1)):
            gh, gl, gr, gc = ctx.encode(img, mb.make_params(**kw), allowed_modes=modes)
            oh, ol, orr, osev, owev = orc.encode(img, orc.make_params(**kw), allowed_modes=modes)
            assert bytes(gh) == bytes(oh) and gl.tobytes() == ol.tobytes()
            assert gr.tobytes() == orr.tobytes() and (gc.search_evals, gc.warmup_evals) == (osev, owev)
            data = mb.format_write(gh, gl, gr)
            h2, l2, r2 = mb.format_read(data)
            assert l2.tobytes() == gl.tobytes() and r2.tobytes() == gr.tobytes()
            dec = ctx.decode(h2, l2, 10, r2)
            assert dec.shape == (h, w)
            assert np.array_equal(dec, orc.decode(oh, ol, 10, orr))


@pytest.mark.gpu
def test_colour_8x8_420_round_trip():
    from mars_b200 import color
    rgb = np.stack([xorshift_plane(8, 8), xorshift_plane(8, 8)[::-1], xorshift_plane(8, 8).T],
                   axis=-1).copy()
    p = mb.make_params(min_size=4, max_size=4, shift=4, lam=2.0)
    with mb.Context(0) as ctx:
        data, _ = color.encode_color(ctx, rgb, color.ColorEncodeParams(p, p))
        out = color.decode_color(ctx, data, 10)
        assert out.shape == (8, 8, 3)
