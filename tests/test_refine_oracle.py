"""The refinement model's FP64 restatement in the oracle: its adjoint gradients against
central finite differences of its own forward fixed point (the check the GPU gradients are
then held to), on encoder-produced leaf lists (modes 0-3, residuals) and on random maps.

The model clamps to 0..255 like the decoder, which puts kinks in the loss where a pixel
sits exactly on a bound (a flat leaf at qbeta = max decodes to exactly 255); a central
difference across a kink is one-sided, so the planes here keep to mid-range grey levels."""
import numpy as np
import pytest

from mars_b200 import synthetic
from oracle import oracle as orc


def _midrange(w, h, seed):
    return (40 + (synthetic.gray(w, h, seed).astype(np.uint32) * 5) // 8).astype(np.uint8)


def _encoded(w, h, seed, modes):
    img = _midrange(w, h, seed)
    hdr, leaves, res, _, _ = orc.encode(img, orc.make_params(min_size=4, max_size=16, shift=4,
                                                             lam=100.0),
                                        allowed_modes=modes)
    return img, hdr, leaves, res


def _random(w, h, seed):
    img = _midrange(w, h, seed + 100)
    leaves = synthetic.quadtree_leaves(w, h, seed, max_size=16, min_size=4)
    leaves["qbeta"] = np.clip(leaves["qbeta"], 16, 100)
    return img, orc.Header(4, 7, 4, 16, 2, w, h, 32), leaves, None


def _fd_check(img, hdr, leaves, res, n_coef=64, h=1e-3, seed=0):
    s, o = orc.refine_params(hdr, leaves)
    loss, _, gs, go = orc.refine_eval(hdr, leaves, img, s, o, res, fwd_iters=500, adj_iters=500)
    rng = np.random.default_rng(seed)
    dom = np.flatnonzero(s > 0)
    flat = np.flatnonzero((s == 0) & (leaves["mode"] != 1))
    picks = [("s", k) for k in rng.choice(dom, min(len(dom), n_coef // 2), replace=False)]
    picks += [("o", k) for k in rng.choice(np.concatenate([dom, flat]), n_coef - len(picks),
                                           replace=False)]
    scale = max(np.abs(gs).max(), np.abs(go).max())
    for which, k in picks:
        sp, sm, op, om = s.copy(), s.copy(), o.copy(), o.copy()
        (sp if which == "s" else op)[k] += h
        (sm if which == "s" else om)[k] -= h
        lp = orc.refine_eval(hdr, leaves, img, sp, op, res, fwd_iters=500, adj_iters=0)[0]
        lm = orc.refine_eval(hdr, leaves, img, sm, om, res, fwd_iters=500, adj_iters=0)[0]
        fd = (lp - lm) / (2 * h)
        an = (gs if which == "s" else go)[k]
        # Central differences carry O(h^2) truncation (the fixed point is rational in s; it
        # is linear in o, so the o checks are exact up to rounding) and loss*eps/h rounding.
        tol = (3e-4 if which == "s" else 1e-6) * abs(an) + 1e-6 * scale + 1e-9 * loss / h
        assert abs(fd - an) <= tol, (which, k, fd, an)
    return loss


@pytest.mark.parametrize("seed,modes", [(1, (1, 0, 1, 0)), (2, (1, 1, 1, 1))])
def test_gradient_vs_central_differences_encoded(seed, modes):
    img, hdr, leaves, res = _encoded(64, 64, seed, modes)
    if modes[3]:
        assert (leaves["mode"] == 3).any()
    _fd_check(img, hdr, leaves, res, seed=seed)


def test_gradient_vs_central_differences_random_map():
    img, hdr, leaves, res = _random(64, 48, 3)
    _fd_check(img, hdr, leaves, res, seed=3)


def test_fixed_point_matches_exact_decode_within_rounding():
    # The continuous model's fixed point is the decoder's attractor up to the rounding of
    # each step: the gap stays within a few grey levels.
    img, hdr, leaves, res = _encoded(64, 64, 4, (1, 1, 1, 1))
    s, o = orc.refine_params(hdr, leaves)
    _, x, _, _ = orc.refine_eval(hdr, leaves, img, s, o, res, fwd_iters=300, adj_iters=0)
    dec = orc.decode(hdr, leaves, 30, res).astype(np.float64)
    assert np.abs(x - dec).mean() < 1.0
    assert np.abs(x - dec).max() < 16.0


def test_adjoint_without_domains_is_the_plain_residual():
    # Flat leaves only: x* = o, so dL/do_L = sum over L of 2 (o_L - t).
    w = h = 32
    rows = [(r, c, 8, 0, 0, 40 + r + c, 0, 0, 0, 0, 0) for r in range(0, h, 8) for c in range(0, w, 8)]
    leaves = np.array(rows, dtype=orc.LEAF_DTYPE)
    hdr = orc.Header(4, 7, 4, 16, 2, w, h, 32)
    img = synthetic.gray(w, h, 9)
    s, o = orc.refine_params(hdr, leaves)
    loss, x, gs, go = orc.refine_eval(hdr, leaves, img, s, o, fwd_iters=3, adj_iters=3)
    for k, L in enumerate(leaves):
        blk = img[L["row"]:L["row"] + 8, L["col"]:L["col"] + 8].astype(np.float64)
        assert go[k] == pytest.approx(np.sum(2 * (o[k] - blk)), rel=1e-12)
    assert np.all(gs == 0)


def test_oracle_search_takes_a_foreign_domain_pool():
    # The cross-plane oracle of the attractor re-search: the plane's own contraction passed
    # in gives the plain search; another plane's contraction gives that plane's domains.
    import numpy as np
    from mars_b200 import synthetic
    from oracle import oracle as orc
    t = synthetic.gray(48, 48, 5)
    x = synthetic.gray(48, 48, 6)
    p = orc.make_params(shift=2)
    for r, c in [(0, 0), (8, 24), (40, 40)]:
        a, ea = orc.search(t, r, c, 8, 2, p)
        b, eb = orc.search(t, r, c, 8, 2, p, contracted=orc.contract(t))
        assert a.tobytes() == b.tobytes() and ea == eb
        d, _ = orc.search(t, r, c, 8, 2, p, contracted=orc.contract(x))
        assert d[0]["t0"] == a[0]["t0"] and d[0]["t2"] == a[0]["t2"]  # the same range block
