"""The classified colour workload (768x512 RGB from the synthetic generator with a random
channel mix, BT.601 Y + 4:2:0 Cb/Cr, Fisher-classified search, ranges 16..4, domain stride
2, lambda 200) against the oracle.

At full size: the colour planes on the device equal the oracle's (metrics.rs:377-432,
color.rs:60-83), and every node of every plane gets the oracle's Fisher candidate and eval
count (crates/mars-search/src/lib.rs:211-297, 471-552).  Whole RD encodes through the
Fisher provider (whose warm-up walk searches exhaustively) are compared on a 192x128 crop
of the same generator, plane by plane and as MARC bytes."""
import numpy as np
import pytest

import mars_b200 as mb
from mars_b200 import color, synthetic
from oracle import oracle as orc
from tests.test_gpu_fisher import _table_parity

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = mb.Context(0)
    yield c
    c.close()


def _planes(ctx, rgb):
    y, cb, cr = ctx.ycbcr(rgb[..., 0], rgb[..., 1], rgb[..., 2])
    oy, ocb, ocr = orc.ycbcr(rgb[..., 0], rgb[..., 1], rgb[..., 2])
    assert np.array_equal(y, oy) and np.array_equal(cb, ocb) and np.array_equal(cr, ocr)
    cb2, cr2 = ctx.downsample_box(cb), ctx.downsample_box(cr)
    assert np.array_equal(cb2, orc.downsample_box(ocb)) and np.array_equal(cr2, orc.downsample_box(ocr))
    return y, cb2, cr2


@pytest.mark.parametrize("seed", [1, 2])
def test_full_size_planes_and_every_fisher_node(ctx, seed):
    rgb = synthetic.rgb(768, 512, seed)
    y, cb, cr = _planes(ctx, rgb)
    assert y.shape == (512, 768) and cb.shape == (256, 384)
    for plane in (y, cb, cr):
        assert _table_parity(ctx, plane, 4, 16, 2, (4, 8, 16)) > 0


def test_reduced_colour_encode_through_fisher(ctx):
    rgb = synthetic.rgb(192, 128, 3)
    kw = dict(min_size=4, max_size=16, shift=2, lam=200.0)
    params = color.ColorEncodeParams(mb.make_params(**kw), mb.make_params(**kw), method="fisher")
    data, stats = color.encode_color(ctx, rgb, params)
    y, cb, cr = _planes(ctx, rgb)
    streams = []
    for plane in (y, cb, cr):
        h, l, res, sev, _ = orc.encode(plane, orc.make_params(**kw), allowed_modes=(1, 1, 1, 1),
                                       method="fisher")
        streams.append(mb.format_write(mb.Header(*[getattr(h, f) for f, _ in h._fields_]), l, res))
    assert data == color.write_container(color.MODE_RGB_420, streams)
    assert (stats.y_bytes, stats.cb_bytes, stats.cr_bytes) == tuple(len(s) for s in streams)
    out = color.decode_color(ctx, data, 10)
    assert out.shape == rgb.shape


@pytest.mark.parametrize("side,seed", [(256, 1), (384, 6)])
def test_device_buckets_equal_the_reference_c_classifier(ctx, side, seed):
    """The device's classified search reads, for every range block, the bucket the
    reference's own 1998 C classifier assigns (oracle/_ref/libmars1_fisher.so): its eval
    count is that bucket's length and its winner lies in that bucket with isometry
    MAPPING[range iso][domain iso].  Square planes: the C contraction is the intended one."""
    from tests.test_fisher_ref_pin import MAPPING, expected_reads
    img = synthetic.gray(side, side, seed)
    prov = ctx.search_provider(img, mb.make_params(min_size=4, max_size=16, shift=2),
                               method="fisher")
    try:
        for size in (4, 8, 16):
            rows, cols, eff, length, risos, bucket, diso = expected_reads(img, size, 2)
            cands, evals = prov.search_many(rows, cols, size, 2)
            assert np.array_equal(evals, length), size
            ncol = (side - 2 * size) // 2 + 1
            pos = (cands["dom_row"] // 2) * ncol + cands["dom_col"] // 2
            assert cands["valid"].all()
            assert np.array_equal(bucket[pos], eff), size
            assert np.array_equal(cands["isometry"], MAPPING[risos, diso[pos]]), size
    finally:
        prov.close()
