"""Fisher's classified search on the GPU (IndexedSearchProvider with Fisher,
crates/mars-search/src/{lib,fisher,classify,tables}.rs) against the oracle's restatement,
bit-exact: every node's candidate (domain, isometry, qalfa, qbeta, rms bits, moments) and
eval count, and whole encodes through the Fisher provider.

The device classifies from exact integer quadrant sums and a permutation of the quadrants;
the oracle follows the reference literally (f64 blocks, flips, variance_2 loops), so
agreement checks the two formulations against each other."""
import numpy as np
import pytest

import mars_b200 as mb
from mars_b200 import synthetic
from oracle import oracle as orc
from tests.golden_data import fixture_images

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = mb.Context(0)
    yield c
    c.close()


def _grid(w, h, size):
    r, c = np.meshgrid(np.arange(0, h - size + 1, size), np.arange(0, w - size + 1, size),
                       indexing="ij")
    return r.ravel().astype(np.uint32), c.ravel().astype(np.uint32)


def _border_twos(w, h):
    """Size-2 nodes a walk reaches: in-plane children of size-4 nodes that cross the border
    (forced splits, encode.rs:1330-1468)."""
    rows, cols = [], []
    for pr in range(0, h, 4):
        for pc in range(0, w, 4):
            if pr + 4 <= h and pc + 4 <= w:
                continue
            for r in (pr, pr + 2):
                for c in (pc, pc + 2):
                    if r + 2 <= h and c + 2 <= w:
                        rows.append(r)
                        cols.append(c)
    return np.array(rows, np.uint32), np.array(cols, np.uint32)


def _table_parity(ctx, img, min_size, max_size, shift, sizes):
    h, w = img.shape
    prov = ctx.search_provider(img, mb.make_params(min_size=min_size, max_size=max_size,
                                                   shift=shift), method="fisher")
    p = orc.make_params(min_size=min_size, max_size=max_size, shift=shift)
    checked = 0
    for size in sizes:
        # Every in-plane aligned node of size >= min_size is requested by some walk; below
        # min_size only the border nodes that forced splits reach.
        rows, cols = _grid(w, h, size) if size >= min_size else _border_twos(w, h)
        if len(rows) == 0:
            continue
        g, gev = prov.search_many(rows, cols, size, shift)
        o, oev = orc.fisher_search_blocks(img, size, shift, p, rows, cols)
        assert np.array_equal(gev, oev), f"size {size}: eval counts differ"
        assert g.tobytes() == o.tobytes(), f"size {size}: candidates differ"
        checked += len(rows)
    prov.close()
    return checked


@pytest.mark.parametrize("path", ["auto", "simt"])
@pytest.mark.parametrize("shift", [2, 4])
def test_synthetic_plane_every_node(ctx, shift, path):
    # "simt" runs every size on the CUDA-core kernel: 1, 2 and 4 warps per range block.
    img = synthetic.gray(128, 96, 3)
    ctx.set_search_path(path)
    try:
        assert _table_parity(ctx, img, 4, 32, shift, (4, 8, 16, 32)) > 0
    finally:
        ctx.set_search_path("auto")


@pytest.mark.parametrize("name", ["mixed_129x127", "flat128", "checker8", "noise_u8", "zoneplate",
                                  "ramp_h"])
def test_fixture_images_every_node(ctx, name):
    imgs, _ = fixture_images()
    img = imgs[name]
    h, w = img.shape
    # Unaligned borders index sizes down to 2 (lib.rs:426-458); flat planes leave all but one
    # bucket empty, exercising the first-non-empty fallback (fisher.rs:42-54).
    sizes = (2, 4, 8, 16) if (w % 4 or h % 4) else (4, 8, 16)
    assert _table_parity(ctx, img, 4, 16, 2, sizes) > 0


def test_plane_without_domains(ctx):
    img = synthetic.gray(12, 12, 1)
    prov = ctx.search_provider(img, mb.make_params(min_size=4, max_size=8, shift=2),
                               method="fisher")
    out = prov.search(0, 0, 8, 2)
    assert out.candidate is None and out.evals == 0
    prov.close()


def _encode_parity(ctx, img, params_kw, modes, adaptive=False):
    gh, gl, gr, gc = ctx.encode(img, mb.make_params(**params_kw), allowed_modes=modes,
                                adaptive_density=adaptive, method="fisher")
    oh, ol, orr, osev, owev = orc.encode(img, orc.make_params(**params_kw), allowed_modes=modes,
                                         adaptive_density=adaptive, method="fisher")
    assert bytes(gh) == bytes(oh)
    assert (gc.search_evals, gc.warmup_evals) == (osev, owev)
    assert gl.tobytes() == ol.tobytes()
    assert gr.tobytes() == orr.tobytes()
    return gc


@pytest.mark.parametrize("lam", [None, 50.0, 200.0])
def test_fisher_encodes(ctx, lam):
    # encmars --method fisher (IndexedSearchProvider::build with Fisher): the final walk
    # searches the Fisher index, the RD warm-up stays exhaustive.
    img = synthetic.gray(128, 128, 7)
    gc = _encode_parity(ctx, img, dict(min_size=4, max_size=16, shift=2, lam=lam), (1, 1, 1, 1))
    ex = ctx.encode(img, mb.make_params(min_size=4, max_size=16, shift=2, lam=lam),
                    allowed_modes=(1, 1, 1, 1))[3]
    assert gc.search_evals < ex.search_evals / 50
    assert gc.warmup_evals == ex.warmup_evals


def test_fisher_encode_adaptive_density_and_borders(ctx):
    imgs, _ = fixture_images()
    _encode_parity(ctx, imgs["mixed_129x127"], dict(min_size=4, max_size=16, shift=2, lam=200.0),
                   (1, 1, 1, 0), adaptive=True)
    _encode_parity(ctx, imgs["mixed_250x250"], dict(min_size=4, max_size=32, shift=4, t_rms=8.0),
                   (1, 0, 1, 0))


@pytest.mark.parametrize("name,side,seed", [("synthetic", 256, 11), ("synthetic", 384, 12),
                                            ("flat128", 0, 0), ("checker8", 0, 0)])
def test_tensor_core_batch_equals_cuda_core_kernel(ctx, name, side, seed):
    """The class-bucketed tcgen05 batch (sizes 4, 8, 16) and the CUDA-core Fisher kernel give
    the same node table bit for bit: same winners, rms bits, moments and eval counts; flat128
    sends every range to one bucket (the first-non-empty fallback) and checker8 to few."""
    if name == "synthetic":
        img = synthetic.gray(side, side, seed)
    else:
        img = fixture_images()[0][name]
    h, w = img.shape
    params = mb.make_params(min_size=4, max_size=16, shift=2)
    simt = mb.Context(0)
    simt.set_search_path("simt")
    try:
        a = ctx.search_provider(img, params, method="fisher")
        b = simt.search_provider(img, params, method="fisher")
        for size in (4, 8, 16):
            rows, cols = _grid(w, h, size)
            x, xe = a.search_many(rows, cols, size, 2)
            y, ye = b.search_many(rows, cols, size, 2)
            assert np.array_equal(xe, ye), size
            assert x.tobytes() == y.tobytes(), size
        a.close()
        b.close()
    finally:
        simt.close()


@pytest.mark.parametrize("w,h", [(768, 512), (384, 256), (129, 127)])
def test_fisher_plan_tables_equal_the_provider(ctx, w, h):
    # mars_indexed_plan_create with Fisher: the graph-captured classified search, run on
    # several planes of one geometry (host and device entry points), gives the one-shot
    # provider's candidates and per-node eval counts (the bucket lengths of each plane).
    import torch
    p = mb.make_params(min_size=4, max_size=16, shift=2, lam=200.0)
    plan = ctx.search_plan(w, h, p, method="fisher")
    try:
        for seed in (1, 2, 3):
            img = synthetic.gray(w, h, seed)
            want = ctx.search_provider(img, p, method="fisher")
            if seed == 3:
                d = torch.from_numpy(img).cuda()
                torch.cuda.synchronize()
                plan.run_device(d.data_ptr())
                got = plan.table()
            else:
                got = plan.run(img)
            sizes = (16, 8, 4) + ((2,) if (w % 4 or h % 4) else ())
            for size in sizes:
                rows, cols = _grid(w, h, size) if size >= 4 else _border_twos(w, h)
                if len(rows) == 0:
                    continue
                a, ae = got.search_many(rows, cols, size, 2)
                b, be = want.search_many(rows, cols, size, 2)
                assert a.tobytes() == b.tobytes(), (seed, size)
                assert np.array_equal(ae, be), (seed, size)
            assert plan.evals == int(mb.lib().mars_search_table_evals(want._h))
            got.close()
            want.close()
    finally:
        plan.close()


def test_fisher_plan_refuses_planned_encodes(ctx):
    plan = ctx.search_plan(64, 64, mb.make_params(min_size=4, max_size=16, shift=2, lam=200.0),
                           method="fisher")
    try:
        with pytest.raises(mb.MarsError):
            plan.encode(synthetic.gray(64, 64, 1))
    finally:
        plan.close()


@pytest.mark.parametrize("lam", [None, 200.0])
def test_fisher_encodes_through_cached_plans(ctx, lam):
    # From a geometry's second Fisher encode on, mars_encode serves the final walk from the
    # context's Fisher search plan and the warm-up walk from its exhaustive plan: the
    # results stay the oracle's, plane after plane.
    kw = dict(min_size=4, max_size=16, shift=2, lam=lam)
    for seed in (11, 12, 13):
        _encode_parity(ctx, synthetic.gray(96, 64, seed), kw, (1, 1, 1, 1))
