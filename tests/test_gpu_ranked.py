"""The ranked provider (SearchProvider::search_candidates over search_top_k,
encode.rs:561-601, 676-788) and rd_candidates encodes on the GPU against the oracle,
bit-exact: every node's best k candidates in (rms, reference order), and whole RD encodes
whose modes 2/3 compete over those lists."""
import numpy as np
import pytest

import mars_b200 as mb
from mars_b200 import synthetic
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = mb.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("k", [2, 3, 8])
def test_ranked_table_every_node(ctx, k):
    img = synthetic.gray(96, 80, 31 + k)
    kw = dict(min_size=4, max_size=16, shift=2)
    prov = ctx.search_provider(img, mb.make_params(**kw), k=k)
    p = orc.make_params(**kw)
    for size in (4, 8, 16):
        for r in range(0, 80 - size + 1, size):
            for c in range(0, 96 - size + 1, size):
                got, gev = prov.search_candidates(r, c, size, 2, k)
                want, oev = orc.search(img, r, c, size, 2, p, k=k)
                assert gev == oev
                assert got.tobytes() == want.tobytes(), (r, c, size)
                head, _ = prov.search_candidates(r, c, size, 2, 1)
                assert head.tobytes() == want[:1].tobytes()
    prov.close()


def test_single_winner_tables_answer_one(ctx):
    img = synthetic.gray(64, 64, 40)
    prov = ctx.search_provider(img, mb.make_params(min_size=4, max_size=16, shift=4))
    got, ev = prov.search_candidates(0, 0, 8, 4, 5)
    assert len(got) == 1 and got[0]["valid"] == 1
    prov.close()
    with pytest.raises(ValueError):
        ctx.search_provider(img, mb.make_params(), method="fisher", k=2)
    with pytest.raises(mb.MarsError):
        ctx.search_provider(img, mb.make_params(), k=9)


@pytest.mark.parametrize("k,modes", [(3, (1, 0, 1, 1)), (8, (1, 1, 1, 1)), (2, (1, 0, 1, 0))])
def test_rd_candidates_encodes(ctx, k, modes):
    img = synthetic.gray(128, 96, 41)
    kw = dict(min_size=4, max_size=16, shift=2, lam=200.0)
    gh, gl, gr, gc = ctx.encode(img, mb.make_params(**kw), allowed_modes=modes, rd_candidates=k)
    oh, ol, orr, osev, owev = orc.encode(img, orc.make_params(**kw), allowed_modes=modes,
                                         rd_candidates=k)
    assert bytes(gh) == bytes(oh)
    assert (gc.search_evals, gc.warmup_evals) == (osev, owev)
    assert gl.tobytes() == ol.tobytes() and gr.tobytes() == orr.tobytes()
    one = ctx.encode(img, mb.make_params(**kw), allowed_modes=modes)
    assert gc.search_evals == one[3].search_evals


def test_rd_candidates_preconditions(ctx):
    img = synthetic.gray(32, 32, 42)
    with pytest.raises(mb.MarsError, match="RD path"):
        ctx.encode(img, mb.make_params(min_size=4, max_size=16, shift=4), rd_candidates=2)
    with pytest.raises(mb.MarsError, match="exhaustive"):
        ctx.encode(img, mb.make_params(min_size=4, max_size=16, shift=4, lam=200.0),
                   rd_candidates=2, method="fisher")


@pytest.mark.parametrize("name,w,h,shift,max_size,k", [
    ("synthetic", 256, 192, 2, 32, 3), ("synthetic", 384, 256, 4, 64, 8),
    ("synthetic", 129, 127, 2, 16, 2), ("flat128", 0, 0, 2, 16, 8),
    ("checker8", 0, 0, 2, 32, 5), ("noise_u8", 0, 0, 8, 32, 4)])
def test_tensor_core_ranked_equals_cuda_core_ranked(ctx, name, w, h, shift, max_size, k):
    # The ranked search runs on the tcgen05 kernel (sizes 4 and 8 on the fold path, 16..64 on
    # the split-digit path: per range a sorted k-list in shared memory, pruned against its
    # k-th entry, seeded with the best k distinct of the 72 seed candidates) and on the
    # CUDA-core kernel: the same k candidates, rms bits, moments and eval counts per node.
    # flat128 makes every candidate tie (queue overflows and re-scans from the first tile).
    from tests.golden_data import fixture_images
    img = synthetic.gray(w, h, 50 + k) if name == "synthetic" else fixture_images()[0][name]
    hh, ww = img.shape
    params = mb.make_params(min_size=4, max_size=max_size, shift=shift)
    simt = mb.Context(0)
    simt.set_search_path("simt")
    try:
        a = ctx.search_provider(img, params, k=k)
        b = simt.search_provider(img, params, k=k)
        checked = 0
        for size in (64, 32, 16, 8, 4):
            if size > max_size:
                continue
            for r in range(0, hh - size + 1, size):
                for c in range(0, ww - size + 1, size):
                    x, xe = a.search_candidates(r, c, size, shift, k)
                    y, ye = b.search_candidates(r, c, size, shift, k)
                    assert xe == ye and x.tobytes() == y.tobytes(), (r, c, size)
                    checked += 1
        assert checked > 0
        a.close()
        b.close()
    finally:
        simt.close()


def test_tensor_core_ranked_equals_oracle_at_stride_4():
    img = synthetic.gray(160, 128, 61)
    kw = dict(min_size=4, max_size=32, shift=4)
    c = mb.Context(0)
    try:
        prov = c.search_provider(img, mb.make_params(**kw), k=4)
        p = orc.make_params(**kw)
        for size in (32, 16, 8, 4):
            for r in range(0, 128 - size + 1, size):
                for col in range(0, 160 - size + 1, size):
                    got, gev = prov.search_candidates(r, col, size, 4, 4)
                    want, oev = orc.search(img, r, col, size, 4, p, k=4)
                    assert gev == oev and got.tobytes() == want.tobytes(), (r, col, size)
        prov.close()
    finally:
        c.close()
