"""Graph-captured search plans (mars_search_plan_*): every replay gives the table the
one-shot provider factory builds for the same plane, bit for bit, through both the host and
the device entry points; tables outlive their plan."""
import numpy as np
import pytest

import mars_b200 as mb
from mars_b200 import synthetic

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = mb.Context(0)
    yield c
    c.close()


def _nodes(w, h, sizes):
    for size in sizes:
        for r in range(0, h - size + 1, size):
            for c in range(0, w - size + 1, size):
                yield r, c, size


def _same(a, b, w, h, sizes, shift):
    for r, c, size in _nodes(w, h, sizes):
        x, y = a.search(r, c, size, shift), b.search(r, c, size, shift)
        assert x == y, (r, c, size)


@pytest.mark.parametrize("w,h", [(128, 96), (200, 136)])
def test_replays_match_the_factory(ctx, w, h):
    params = mb.make_params(min_size=4, max_size=32, shift=2, lam=200.0)
    plan = ctx.search_plan(w, h, params)
    assert plan.launches > 0
    for seed in (1, 2, 3):
        img = synthetic.gray(w, h, seed)
        got = plan.run(img)
        want = ctx.search_provider(img, params)
        assert mb.lib().mars_search_table_evals(got._h) == mb.lib().mars_search_table_evals(want._h)
        _same(got, want, w, h, (4, 8, 16, 32), 2)
        got.close()
        want.close()
    plan.close()


def test_device_replays_and_tables_outlive_the_plan(ctx):
    import torch
    w, h = 160, 128
    params = mb.make_params(min_size=4, max_size=16, shift=4)
    plan = ctx.search_plan(w, h, params)
    img = synthetic.gray(w, h, 7)
    d = torch.from_numpy(img).to("cuda:0")
    torch.cuda.synchronize()
    plan.run_device(d.data_ptr())
    t = plan.table()
    plan.close()
    want = ctx.search_provider(img, params)
    _same(t, want, w, h, (4, 8, 16), 4)
    t.close()
    want.close()


def test_plan_rejects_a_wrong_shape(ctx):
    plan = ctx.search_plan(64, 64, mb.make_params(min_size=4, max_size=16, shift=2))
    with pytest.raises(ValueError):
        plan.run(np.zeros((32, 64), np.uint8))
    plan.close()


@pytest.mark.parametrize("modes,lam", [((1, 0, 1, 0), 200.0), ((1, 1, 1, 1), 50.0), ((1, 0, 1, 0), None)])
def test_planned_encodes_equal_the_one_shot_encode(ctx, modes, lam):
    params = mb.make_params(min_size=4, max_size=16, shift=2, lam=lam)
    imgs = [synthetic.gray(96, 80, s) for s in (3, 4, 5, 6)] + [synthetic.gray(64, 64, 7)]
    many = ctx.encode_many(imgs, params, workers=3, allowed_modes=modes)
    for im, got in zip(imgs, many):
        want = ctx.encode(im, params, allowed_modes=modes)
        assert bytes(got[0]) == bytes(want[0])
        assert got[1].tobytes() == want[1].tobytes() and got[2].tobytes() == want[2].tobytes()
        assert (got[3].search_evals, got[3].warmup_evals) == (want[3].search_evals,
                                                              want[3].warmup_evals)


def test_planned_encode_refuses_what_a_plan_cannot_serve(ctx):
    params = mb.make_params(min_size=4, max_size=16, shift=2, lam=200.0)
    plan = ctx.search_plan(64, 64, params)
    img = synthetic.gray(64, 64, 8)
    opts = mb.Options((mb.C.c_uint8 * 4)(1, 0, 1, 0), 0, 0, 0.0, 1, 1)  # Fisher
    hdr, cnt = mb.Header(), mb.Counters()
    ptr, n, rptr, rn = mb.C.c_void_p(), mb.C.c_size_t(), mb.C.c_void_p(), mb.C.c_size_t()
    rc = mb.lib().mars_encode_planned(plan._h, img.ctypes.data, mb.C.byref(opts), mb.C.byref(hdr),
                                      mb.C.byref(ptr), mb.C.byref(n), mb.C.byref(rptr),
                                      mb.C.byref(rn), mb.C.byref(cnt))
    assert rc == -8  # MARS_EUNSUPPORTED
    plan.close()


def _grid(w, h, size):
    r, c = np.meshgrid(np.arange(0, h - size + 1, size), np.arange(0, w - size + 1, size),
                       indexing="ij")
    return r.ravel().astype(np.uint32), c.ravel().astype(np.uint32)


@pytest.mark.parametrize("w,h,shift,max_size", [(512, 512, 2, 32), (200, 136, 2, 32),
                                                (129, 127, 4, 16), (256, 256, 8, 64),
                                                (384, 320, 16, 64), (96, 64, 2, 8)])
def test_all_levels_launch_equals_per_level_launches(ctx, w, h, shift, max_size):
    # Tables and plans correlate every tensor-core level in one persistent launch (work items
    # of every level from one counter, pipelines carried from item to item, each range tile
    # finished by its last split); one launch per level gives the same candidates, rms bits
    # and moments for every node, and fewer kernel launches are made.
    img = synthetic.gray(w, h, 5)
    params = mb.make_params(min_size=4, max_size=max_size, shift=shift, lam=200.0)
    per = mb.Context(0)
    per.set_search_path("per_level")
    try:
        a = ctx.search_provider(img, params)
        b = per.search_provider(img, params)
        plan = ctx.search_plan(w, h, params)
        per_plan = per.search_plan(w, h, params)
        got = plan.run(img)
        for size in (64, 32, 16, 8, 4):
            if size > max_size:
                continue
            rows, cols = _grid(w, h, size)
            if len(rows) == 0:
                continue
            x, xe = a.search_many(rows, cols, size, shift)
            y, ye = b.search_many(rows, cols, size, shift)
            z, ze = got.search_many(rows, cols, size, shift)
            assert x.tobytes() == y.tobytes(), size
            assert z.tobytes() == y.tobytes(), size
            assert np.array_equal(xe, ye) and np.array_equal(ze, ye), size
        assert plan.launches < per_plan.launches
        assert plan.kernel_ms > 0.0  # events recorded around the launch inside the graph
        with pytest.raises(mb.MarsError):
            per_plan.kernel_ms
        for t in (a, b, got):
            t.close()
        plan.close()
        per_plan.close()
    finally:
        per.close()
