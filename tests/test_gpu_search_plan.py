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
