"""The attractor-refinement kernels (mars_refine_*) against the oracle's FP64 restatement of
the same model: the fixed point, the loss and the adjoint gradients; then the refinement
loop end to end (re-quantised leaves that decode exactly, kept only when they decode
better, still writable as .mars)."""
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


def _midrange(w, h, seed):
    return (40 + (synthetic.gray(w, h, seed).astype(np.uint32) * 5) // 8).astype(np.uint8)


def _mb_hdr(oh):
    return mb.Header(*[getattr(oh, f) for f, _ in oh._fields_])


def _psnr(a, b):
    mse = np.mean((a.astype(np.float64) - b.astype(np.float64)) ** 2)
    return 10 * np.log10(255.0 ** 2 / mse)


CASES = [("encoded", 96, 64, 1, (1, 0, 1, 0)), ("encoded", 64, 64, 2, (1, 1, 1, 1)),
         ("random", 128, 96, 3, None)]


def _case(kind, w, h, seed, modes):
    img = _midrange(w, h, seed)
    if kind == "encoded":
        oh, leaves, res, _, _ = orc.encode(img, orc.make_params(min_size=4, max_size=16, shift=4,
                                                                lam=100.0),
                                           allowed_modes=modes)
        return img, oh, leaves, res
    leaves = synthetic.quadtree_leaves(w, h, seed, max_size=16, min_size=4)
    leaves["qbeta"] = np.clip(leaves["qbeta"], 16, 100)
    return img, orc.Header(4, 7, 4, 16, 2, w, h, 32), leaves, None


@pytest.mark.parametrize("kind,w,h,seed,modes", CASES)
def test_forward_and_gradients_match_fp64(ctx, kind, w, h, seed, modes):
    img, oh, leaves, res = _case(kind, w, h, seed, modes)
    plan = ctx.refine_plan(_mb_hdr(oh), leaves, img, res)
    s, o = plan.params()
    so, oo = orc.refine_params(oh, leaves)
    assert np.array_equal(s, so.astype(np.float32)) and np.array_equal(o, oo.astype(np.float32))
    loss, iters, x = plan.forward(s, o, max_iters=1000, tol=1e-4, want_x=True)
    ol, ox, ogs, ogo = orc.refine_eval(oh, leaves, img, s.astype(np.float64), o.astype(np.float64),
                                       res, fwd_iters=800, adj_iters=800)
    # f32 iterates against f64: the fixed points agree to a few f32 ulps of 255 times the
    # contraction's gain.
    assert np.abs(x - ox).max() < 2e-2
    assert loss == pytest.approx(ol, rel=1e-4)
    gs, go, aiters, rel = plan.backward(max_iters=1000, tol=1e-6)
    assert rel < 1e-5
    g = np.concatenate([gs, go]).astype(np.float64)
    og = np.concatenate([ogs, ogo])
    assert np.linalg.norm(g - og) <= 1e-3 * np.linalg.norm(og)
    assert np.all(np.abs(g - og) <= 2e-3 * np.abs(og) + 1e-3 * np.abs(og).max())
    plan.close()


def test_backward_needs_a_forward(ctx):
    img, oh, leaves, res = _case("random", 64, 64, 5, None)
    plan = ctx.refine_plan(_mb_hdr(oh), leaves, img, res)
    with pytest.raises(mb.MarsError, match="forward"):
        plan.backward()
    with pytest.raises(mb.MarsError, match="lr"):
        plan.run(steps=1, lr=0.0)
    with pytest.raises(ValueError):
        ctx.refine_plan(_mb_hdr(oh), leaves, img[:-1], res)
    plan.close()


def test_rejects_invalid_leaves(ctx):
    img, oh, leaves, res = _case("random", 64, 64, 6, None)
    bad = leaves.copy()
    bad["qalfa"][int(np.flatnonzero(bad["mode"] == 2)[0])] = 17
    with pytest.raises(mb.MarsError, match="wider"):
        ctx.refine_plan(_mb_hdr(oh), bad, img)


@pytest.mark.parametrize("side,seed", [(128, 7), (192, 8)])
def test_refinement_loop_end_to_end(ctx, side, seed):
    img = synthetic.gray(side, side, seed)
    hdr, leaves, res, _ = ctx.encode(img, mb.make_params(min_size=4, max_size=32, shift=4,
                                                         lam=100.0),
                                     allowed_modes=(1, 1, 1, 1))
    plan = ctx.refine_plan(hdr, leaves, img, res)
    out, rep = plan.run(steps=12, lr=1.0, decode_iterations=10)
    assert rep.loss_end <= rep.loss_start
    assert rep.psnr_plain == pytest.approx(_psnr(ctx.decode(hdr, leaves, 10, res), img), abs=1e-9)
    # Only qalfa/qbeta of modes 0/2/3 move; geometry, isometries and domains stay.
    for f in ("row", "col", "size", "mode", "isometry", "dom_row", "dom_col", "qgx", "qgy"):
        assert np.array_equal(out[f], leaves[f])
    dec = ctx.decode(hdr, out, 10, res)
    if rep.accepted:
        assert rep.psnr_refined > rep.psnr_plain
        assert _psnr(dec, img) == pytest.approx(rep.psnr_refined, abs=1e-9)
        dom = out["mode"] >= 2
        assert np.all(out["qalfa"][dom] >= 1) and np.all(out["qalfa"][dom] < (1 << hdr.bits_alfa))
    else:
        assert np.array_equal(out, leaves)
    # The result is still a valid .mars stream that reads back to the same leaves.
    h2, l2, r2 = mb.format_read(mb.format_write(hdr, out, res))
    assert np.array_equal(l2, out) and np.array_equal(r2, res)
    plan.close()
