"""Parity of the decode gather (mars_decode, mars_decode_plan_*) against the oracle's
decode_iterative (crates/mars-codec/src/ifs.rs:281-309, 406-484), bit-exact."""
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


def _hdr(w, h, bits_alfa=4, bits_beta=7, int_max_alfa=32):
    return mb.Header(bits_alfa, bits_beta, 4, 32, 2, w, h, int_max_alfa)


def _ohdr(hdr):
    return orc.Header(*[getattr(hdr, f) for f, _ in orc.Header._fields_])


@pytest.mark.parametrize("w,h,seed", [(256, 256, 1), (260, 200, 2), (512, 384, 3), (64, 96, 4)])
def test_synthetic_quadtree_maps(ctx, w, h, seed):
    # Modes 0/1/2, all isometries; (260, 200) leaves a border no leaf covers (written 0).
    leaves = synthetic.quadtree_leaves(w, h, seed)
    hdr = _hdr(w, h)
    for iters in (1, 2, 10):
        assert np.array_equal(ctx.decode(hdr, leaves, iters), orc.decode(_ohdr(hdr), leaves, iters))


@pytest.mark.parametrize("bits_alfa,bits_beta,int_max_alfa", [(2, 5, 32), (6, 9, 64), (16, 16, 255),
                                                               (0, 1, 32)])
def test_header_bit_widths(ctx, bits_alfa, bits_beta, int_max_alfa):
    w = h = 128
    leaves = synthetic.quadtree_leaves(w, h, 7, bits_alfa=bits_alfa, bits_beta=bits_beta)
    hdr = _hdr(w, h, bits_alfa, bits_beta, int_max_alfa)
    assert np.array_equal(ctx.decode(hdr, leaves, 6), orc.decode(_ohdr(hdr), leaves, 6))


def test_unaligned_leaves_one_pixel_cells(ctx):
    # Leaves of size 5 at multiples of 5: the owner map falls back to 1x1 cells.
    w = h = 30
    rng = np.random.default_rng(5)
    rows = []
    for r in range(0, h, 5):
        for c in range(0, w, 5):
            mode = int(rng.integers(0, 3))
            qalfa = int(rng.integers(1, 17)) if mode == 2 else 0
            dr, dc = int(rng.integers(0, h - 10 + 1)), int(rng.integers(0, w - 10 + 1))
            rows.append((r, c, 5, mode, qalfa, int(rng.integers(0, 128)), int(rng.integers(0, 8)),
                         dr if mode == 2 else 0, dc if mode == 2 else 0,
                         int(rng.integers(-80, 81)) if mode == 1 else 0,
                         int(rng.integers(-80, 81)) if mode == 1 else 0))
    leaves = np.array(rows, dtype=mb.LEAF_DTYPE)
    hdr = _hdr(w, h)
    for iters in (1, 4):
        assert np.array_equal(ctx.decode(hdr, leaves, iters), orc.decode(_ohdr(hdr), leaves, iters))


def _mode3(leaves, rng, p_zero=0.5):
    """Turn the domain leaves into mode-3 leaves, half of them with qalfa = 0 (no domain
    read, the residual still added: ifs.rs:459-479), with random residual levels."""
    out = leaves.copy()
    pool = []
    for k in range(len(out)):
        if out["mode"][k] != 2:
            continue
        out["mode"][k] = 3
        if rng.random() < p_zero:
            out["qalfa"][k] = 0
        n = int(out["size"][k]) ** 2
        lv = np.zeros(n, np.int32)
        nz = rng.choice(n, size=min(n, 6), replace=False)
        lv[nz] = rng.integers(-20, 21, size=len(nz))
        pool.append(lv)
    return out, (np.concatenate(pool) if pool else np.zeros(0, np.int32))


@pytest.mark.parametrize("w,h,seed", [(128, 96, 11), (30, 30, 12)])
def test_zero_alpha_residual_leaves(ctx, w, h, seed):
    rng = np.random.default_rng(seed)
    if w == 30:  # size-5 leaves: the one-pixel-cell kernel
        rows = []
        for r in range(0, h, 5):
            for c in range(0, w, 5):
                dr, dc = int(rng.integers(0, h - 9)), int(rng.integers(0, w - 9))
                rows.append((r, c, 5, 2, int(rng.integers(1, 17)), int(rng.integers(0, 128)),
                             int(rng.integers(0, 8)), dr, dc, 0, 0))
        base = np.array(rows, dtype=mb.LEAF_DTYPE)
    else:
        base = synthetic.quadtree_leaves(w, h, seed)
    leaves, pool = _mode3(base, rng)
    assert (leaves["mode"] == 3).any() and ((leaves["mode"] == 3) & (leaves["qalfa"] == 0)).any()
    hdr = _hdr(w, h)
    for iters in (1, 5):
        assert np.array_equal(ctx.decode(hdr, leaves, iters, pool),
                              orc.decode(_ohdr(hdr), leaves, iters, pool))


def test_later_leaves_overwrite_earlier(ctx):
    # decode_step writes leaves in order, so a later leaf wins where two overlap.
    w = h = 64
    base = synthetic.quadtree_leaves(w, h, 9)
    extra = synthetic.quadtree_leaves(w, h, 10, max_size=16)[:20]
    leaves = np.concatenate([base, extra])
    hdr = _hdr(w, h)
    for iters in (1, 5):
        assert np.array_equal(ctx.decode(hdr, leaves, iters), orc.decode(_ohdr(hdr), leaves, iters))


def test_empty_leaf_list_decodes_to_zero(ctx):
    hdr = _hdr(32, 16)
    out = ctx.decode(hdr, np.zeros(0, dtype=mb.LEAF_DTYPE), 3)
    assert out.shape == (16, 32) and not out.any()
    assert np.array_equal(out, orc.decode(_ohdr(hdr), np.zeros(0, dtype=mb.LEAF_DTYPE), 3))


@pytest.mark.parametrize("iters", [0, 1, 2, 7, 10])
def test_decode_plan_matches_decode(ctx, iters):
    import torch
    w, h = 320, 256
    leaves = synthetic.quadtree_leaves(w, h, 11)
    hdr = _hdr(w, h)
    plan = ctx.decode_plan(hdr, leaves)
    dev = torch.empty(w * h, dtype=torch.uint8, device="cuda:0")
    for _ in range(2):  # a plan runs any number of times
        dev.fill_(7)
        torch.cuda.synchronize()
        plan.run(iters, dev.data_ptr())
        torch.cuda.synchronize()
        got = dev.cpu().numpy().reshape(h, w)
        assert np.array_equal(got, ctx.decode(hdr, leaves, iters))
        assert np.array_equal(got, orc.decode(_ohdr(hdr), leaves, iters))
    plan.close()


def test_decode_rejects_out_of_range_leaves(ctx):
    hdr = _hdr(64, 64)
    leaves = synthetic.quadtree_leaves(64, 64, 12)
    k = int(np.flatnonzero(leaves["mode"] == 2)[0])
    bad = leaves.copy()
    bad["qalfa"][k] = 17  # above 2^bits_alfa
    with pytest.raises(mb.MarsError) as e:
        ctx.decode(hdr, bad, 2)
    assert e.value.code == -1
    bad = leaves.copy()
    bad["qbeta"][k] = 128  # above 2^bits_beta - 1
    with pytest.raises(mb.MarsError) as e:
        ctx.decode(hdr, bad, 2)
    assert e.value.code == -1
    bad = leaves.copy()
    bad["mode"][k] = 3  # a mode-3 leaf without its residual levels
    with pytest.raises(mb.MarsError, match="residual pool") as e:
        ctx.decode(hdr, bad, 2)
    assert e.value.code == -1
    bad["mode"][k] = 4
    with pytest.raises(mb.MarsError) as e:
        ctx.decode(hdr, bad, 2)
    assert e.value.code == -1
    with pytest.raises(mb.MarsError) as e:
        ctx.decode_plan(_hdr(70000, 8), np.zeros(0, dtype=mb.LEAF_DTYPE))
    assert e.value.code == -1


@pytest.mark.parametrize("threshold", [0, 1, 3, 255])
def test_until_stable_matches_the_oracle(ctx, threshold):
    # Aligned maps take the 4x4-cell kernel, the size-5 map the one-pixel kernel.
    rng = np.random.default_rng(9)
    maps = [(synthetic.quadtree_leaves(160, 96, 21), 160, 96, None)]
    base = synthetic.quadtree_leaves(128, 96, 22)
    leaves3, pool = _mode3(base, rng, p_zero=0.3)
    maps.append((leaves3, 128, 96, pool))
    rows = []
    for r in range(0, 30, 5):
        for c in range(0, 30, 5):
            rows.append((r, c, 5, 2, int(rng.integers(1, 17)), int(rng.integers(0, 128)),
                         int(rng.integers(0, 8)), int(rng.integers(0, 21)), int(rng.integers(0, 21)),
                         0, 0))
    maps.append((np.array(rows, dtype=mb.LEAF_DTYPE), 30, 30, None))
    for leaves, w, h, res in maps:
        hdr = _hdr(w, h)
        got, used = ctx.decode_until_stable(hdr, leaves, threshold, 40, res)
        want, oused = orc.decode_until_stable(_ohdr(hdr), leaves, threshold, 40, res)
        assert used == oused and np.array_equal(got, want)


def test_plan_until_stable_on_the_device(ctx):
    import torch
    leaves = synthetic.quadtree_leaves(256, 192, 23)
    hdr = _hdr(256, 192)
    plan = ctx.decode_plan(hdr, leaves)
    out = torch.zeros(256 * 192, dtype=torch.uint8, device="cuda:0")
    used = mb.C.c_uint32()
    mb.check(mb.lib().mars_decode_plan_run_until_stable(plan._h, 2, 30, out.data_ptr(),
                                                        mb.C.byref(used)))
    torch.cuda.synchronize()
    want, oused = orc.decode_until_stable(_ohdr(hdr), leaves, 2, 30)
    assert used.value == oused
    assert np.array_equal(out.cpu().numpy().reshape(192, 256), want)
    plan.close()


@pytest.mark.parametrize("factor", [2.0, 1.5, 0.5])
def test_zoomed_decode_matches_the_oracle(ctx, factor):
    img = synthetic.gray(128, 96, 24)
    hdr, leaves, res, _ = ctx.encode(img, mb.make_params(min_size=4, max_size=16, shift=4, lam=200.0),
                                     allowed_modes=(1, 1, 1, 1))
    zh, zl = mb.zoom_leaves(hdr, leaves, factor)
    ozh, ozl = orc.zoom_leaves(_ohdr(hdr), leaves, factor)
    assert zl.tobytes() == ozl.tobytes()
    got = ctx.decode(zh, zl, 10)
    assert got.shape == (round(96 * factor), round(128 * factor))
    assert np.array_equal(got, orc.decode(ozh, ozl, 10))


@pytest.mark.parametrize("w,h,seed", [(320, 256, 11), (1024, 768, 13), (516, 302, 14),
                                      (2500, 300, 15), (2052, 148, 16)])
def test_source_ordered_plan_steps_match_the_oracle(ctx, monkeypatch, w, h, seed):
    """The source-ordered steps large planes take (domain cells gathered in the order of their
    windows' source rows into a cell buffer, then placed in output order) give the cell
    kernel's bytes: forced on here for planes small enough for the oracle; (516, 302) leaves a
    border no leaf covers and a last cell row cut by the plane's edge."""
    import torch
    monkeypatch.setenv("MARS_DECODE_SORTED", "1")
    leaves = synthetic.quadtree_leaves(w, h, seed)
    hdr = _hdr(w, h)
    plan = ctx.decode_plan(hdr, leaves)
    dev = torch.empty(w * h, dtype=torch.uint8, device="cuda:0")
    for iters in (1, 3, 10):
        dev.fill_(7)
        torch.cuda.synchronize()
        plan.run(iters, dev.data_ptr())
        torch.cuda.synchronize()
        got = dev.cpu().numpy().reshape(h, w)
        assert np.array_equal(got, orc.decode(_ohdr(hdr), leaves, iters)), iters
    plan.close()
