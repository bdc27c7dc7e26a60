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


# ---- the domain re-search against the attractor (mars_refine_domains) and the two-plane
# search under it (mars_search_blocks_cross_device)

def _cross_planes(w, h, seed):
    """A target plane and a second plane of the same size standing in for its decode: the
    target with seeded noise and a small shift, so the two pools differ everywhere."""
    t = synthetic.gray(w, h, seed)
    rng = np.random.default_rng(seed)
    x = np.roll(t.astype(np.int32), 1, axis=1) + rng.integers(-9, 10, size=t.shape)
    return t, np.clip(x, 0, 255).astype(np.uint8)


def _cross_device(ctx, t, x, size, shift, p, rows, cols):
    import torch
    h, w = t.shape
    d_t = torch.from_numpy(t).cuda()
    d_x = torch.from_numpy(x).cuda()
    d_r = torch.from_numpy(np.asarray(rows, np.int32)).cuda()
    d_c = torch.from_numpy(np.asarray(cols, np.int32)).cuda()
    out = torch.zeros((len(rows), mb.CANDIDATE_DTYPE.itemsize), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    mb.check(mb.lib().mars_search_blocks_cross_device(ctx.handle, d_t.data_ptr(), d_x.data_ptr(),
                                                      w, h, size, shift, mb.C.byref(p),
                                                      d_r.data_ptr(), d_c.data_ptr(), len(rows),
                                                      out.data_ptr()))
    torch.cuda.synchronize()
    return out.cpu().numpy().view(mb.CANDIDATE_DTYPE).ravel()


@pytest.mark.parametrize("path", ["auto", "simt"])
@pytest.mark.parametrize("size,shift", [(4, 2), (8, 4), (16, 2), (32, 4)])
def test_cross_search_matches_the_oracle(ctx, path, size, shift):
    # Ranges from one plane, domains from another: every aligned block against the oracle's
    # search_top_k over the second plane's contraction, record for record (moments included).
    w, h = 96, 80
    t, x = _cross_planes(w, h, 7 + size)
    rows, cols = np.meshgrid(np.arange(h // size) * size, np.arange(w // size) * size,
                             indexing="ij")
    rows, cols = rows.ravel(), cols.ravel()
    ctx.set_search_path(path)
    try:
        got = _cross_device(ctx, t, x, size, shift, mb.make_params(shift=shift), rows, cols)
    finally:
        ctx.set_search_path("auto")
    cx = orc.contract(x)
    op = orc.make_params(shift=shift)
    for i, (r, c) in enumerate(zip(rows, cols)):
        o, _ = orc.search(t, int(r), int(c), size, shift, op, contracted=cx)
        assert got[i].tobytes() == o[0].tobytes(), (i, r, c)


def test_cross_search_on_one_plane_is_the_search(ctx):
    import torch
    img = synthetic.gray(128, 128, 4)
    rows = np.array([0, 8, 64, 120], np.int32)
    cols = np.array([0, 16, 40, 120], np.int32)
    p = mb.make_params(shift=2)
    got = _cross_device(ctx, img, img, 8, 2, p, rows, cols)
    d_img = torch.from_numpy(img).cuda()
    d_r, d_c = torch.from_numpy(rows).cuda(), torch.from_numpy(cols).cuda()
    out = torch.zeros((4, mb.CANDIDATE_DTYPE.itemsize), dtype=torch.uint8, device="cuda")
    mb.check(mb.lib().mars_search_blocks_device(ctx.handle, d_img.data_ptr(), 128, 128, 8, 2,
                                                mb.C.byref(p), d_r.data_ptr(), d_c.data_ptr(),
                                                4, out.data_ptr()))
    torch.cuda.synchronize()
    assert got.tobytes() == out.cpu().numpy().tobytes()


@pytest.mark.parametrize("seed,lam", [(1, 100.0), (3, 400.0)])
def test_domain_refinement_end_to_end(ctx, seed, lam):
    # Only mode-2 leaves move, to valid domains of the header's grid with qalfa >= 1; the
    # result decodes to the reported PSNR, never below the input's, and stays a valid stream.
    side = 128
    img = synthetic.gray(side, side, seed)
    p = mb.make_params(min_size=4, max_size=32, shift=2, lam=lam)
    hdr, leaves, res, _ = ctx.encode(img, p, allowed_modes=(1, 1, 1, 1))
    out, rep = ctx.refine_domains(p, hdr, leaves, img, res, passes=3, decode_iterations=12)
    for f in ("row", "col", "size", "mode", "qgx", "qgy"):
        assert np.array_equal(out[f], leaves[f]), f
    fixed = leaves["mode"] != 2
    assert out[fixed].tobytes() == leaves[fixed].tobytes()
    moved = out[~fixed]
    assert np.all(moved["qalfa"] >= 1) and np.all(moved["isometry"] < 8)
    assert np.all(moved["dom_row"] % hdr.shift == 0) and np.all(moved["dom_col"] % hdr.shift == 0)
    assert np.all(moved["dom_row"] + 2 * moved["size"] <= side)
    assert np.all(moved["dom_col"] + 2 * moved["size"] <= side)
    p0 = _psnr(ctx.decode(hdr, leaves, 12, res), img)
    p1 = _psnr(ctx.decode(hdr, out, 12, res), img)
    assert rep.psnr_plain == pytest.approx(p0, abs=1e-9)
    assert rep.psnr_refined == pytest.approx(p1, abs=1e-9)
    assert p1 >= p0
    assert rep.changed_leaves == int(np.sum(np.any(
        out.view(np.uint8).reshape(len(out), -1) != leaves.view(np.uint8).reshape(len(out), -1),
        axis=1)))
    assert bool(rep.accepted) == (rep.changed_leaves > 0)
    data = mb.format_write(hdr, out, res)
    h2, l2, r2 = mb.format_read(data)
    assert l2.tobytes() == out.tobytes() and np.array_equal(r2, res)


def test_domain_refinement_with_no_pass_returns_the_input(ctx):
    img = synthetic.gray(64, 64, 2)
    p = mb.make_params(min_size=4, max_size=16, shift=2, lam=200.0)
    hdr, leaves, res, _ = ctx.encode(img, p, allowed_modes=(1, 0, 1, 0))
    out, rep = ctx.refine_domains(p, hdr, leaves, img, res, passes=0)
    assert out.tobytes() == leaves.tobytes()
    assert rep.steps == 0 and rep.accepted == 0 and rep.changed_leaves == 0
