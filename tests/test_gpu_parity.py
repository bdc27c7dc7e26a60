"""Parity of the CUDA path against the CPU oracle, through the C ABI.

The bar is bit-exact: every candidate field (domain, isometry, qalfa, qbeta, the f64 rms
bit pattern and the six integer moments), every leaf and every eval count.
"""
import hashlib

import numpy as np
import pytest

import mars_b200 as mb
from mars_b200 import synthetic
from oracle import oracle as orc
from tests.golden_data import fixture_images, mars1_bytes, mars1_manifest, provider_pattern_16

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = mb.Context(0)
    yield c
    c.close()


def _xorshift_image(seed, h, w):
    s = seed
    out = np.empty(h * w, dtype=np.uint8)
    for i in range(h * w):
        s ^= (s << 13) & 0xFFFFFFFFFFFFFFFF
        s ^= s >> 7
        s ^= (s << 17) & 0xFFFFFFFFFFFFFFFF
        out[i] = s & 0xFF
    return out.reshape(h, w)


def _grid_parity(ctx, img, size, shift, params):
    g, gev = ctx.search_grid(img, size, shift, params)
    o, oev = orc.search_grid(img, size, shift, orc.make_params(
        min_size=params.min_size, max_size=params.max_size, shift=params.shift,
        bits_alfa=params.bits_alfa, bits_beta=params.bits_beta, max_alfa=params.max_alfa))
    assert np.array_equal(gev, oev)
    bad = np.nonzero(g.view(np.uint8).reshape(len(g), -1) != o.view(np.uint8).reshape(len(o), -1))[0]
    if len(bad):
        i = int(bad[0])
        pytest.fail(f"block {i}: gpu {g[i]} != oracle {o[i]} ({len(np.unique(bad))} differ)")


@pytest.mark.parametrize("size", [4, 8, 16])
def test_config1_grid_parity(ctx, size):
    # 256x256 synthetic seed 0, shift 4, sizes 16..4
    img = synthetic.gray(256, 256, 0)
    _grid_parity(ctx, img, size, 4, mb.make_params(shift=4))


@pytest.mark.parametrize("size,shift", [(4, 2), (8, 2), (16, 2), (32, 2), (32, 4), (2, 2), (64, 2)])
def test_shift2_grid_parity_synthetic_crop(ctx, size, shift):
    img = synthetic.gray(512, 512, 1)[:160, :192]
    _grid_parity(ctx, img, size, shift, mb.make_params(shift=shift))


@pytest.mark.parametrize("name", ["flat128", "ramp_h", "checker8", "noise_u8", "impulse",
                                  "step_edge", "selfsim_iso", "zoneplate", "mixed_129x127",
                                  "mixed_250x250"])
def test_fixture_images_grid_parity(ctx, name):
    imgs, _ = fixture_images()
    img = imgs[name]
    for size in (4, 8):
        _grid_parity(ctx, img, size, 4, mb.make_params())


def test_xorshift_random_planes(ctx):
    for seed, (h, w) in [(1, (32, 32)), (7, (40, 24)), (99, (64, 48))]:
        img = _xorshift_image(seed, h, w)
        for size in (2, 4, 8, 16):
            if 2 * size <= min(h, w):
                _grid_parity(ctx, img, size, 2, mb.make_params())


def test_nonunit_max_alfa_and_bits(ctx):
    img = synthetic.gray(96, 96, 5)
    for kw in (dict(max_alfa=0.75), dict(max_alfa=1.5, bits_alfa=5), dict(bits_beta=6),
               dict(max_alfa=2.0, bits_alfa=3, bits_beta=8)):
        p = mb.make_params(**kw)
        g, _ = ctx.search_grid(img, 8, 2, p)
        o, _ = orc.search_grid(img, 8, 2, orc.make_params(**kw))
        assert g.tobytes() == o.tobytes(), kw


def test_no_legal_domain_is_none(ctx):
    img = synthetic.gray(24, 24, 3)
    g, ev = ctx.search_blocks(img, 16, 2, mb.make_params(), [0], [0])
    assert g[0]["valid"] == 0 and ev[0] == 0
    o, oev = orc.search(img, 0, 0, 16, 2, orc.make_params())
    assert len(o) == 0 and oev == 0


def _encode_parity(ctx, img, params_kw, modes=(1, 0, 1, 0), adaptive=False, **resid):
    gh, gl, gr, gc = ctx.encode(img, mb.make_params(**params_kw), allowed_modes=modes,
                                adaptive_density=adaptive, **resid)
    oh, ol, orr, osev, owev = orc.encode(img, orc.make_params(**params_kw), allowed_modes=modes,
                                         adaptive_density=adaptive, **resid)
    assert bytes(gh) == bytes(oh)
    assert (gc.search_evals, gc.warmup_evals) == (osev, owev)
    assert gl.tobytes() == ol.tobytes()
    assert gr.tobytes() == orr.tobytes()
    return gh, gl


def test_provider_pattern_encodes(ctx):
    # crates/mars-codec/tests/search_provider.rs:29-66 (evals 608 / 1184 / 864 / 1184)
    img = provider_pattern_16()
    base = dict(min_size=4, max_size=8, shift=4, t_rms=8.0)
    _encode_parity(ctx, img, base)
    _encode_parity(ctx, img, dict(base, lam=2.0), modes=(1, 1, 1, 1))
    _encode_parity(ctx, img, dict(base, lam=2.0), modes=(1, 1, 1, 1), adaptive=True,
                   residual_adaptive=True)
    _encode_parity(ctx, img, dict(base, lam=50.0), residual_qstep=17.123456789)


@pytest.mark.parametrize("lam", [None, 50.0, 200.0, 800.0])
def test_config1_encode_parity(ctx, lam):
    img = synthetic.gray(256, 256, 0)
    _encode_parity(ctx, img, dict(min_size=4, max_size=16, shift=4, lam=lam))


@pytest.mark.parametrize("lam", [50.0, 200.0])
def test_all_modes_encode_parity(ctx, lam):
    # The reference's default EncodeOptions: all four modes, residual step 8.
    img = synthetic.gray(128, 128, 5)
    _encode_parity(ctx, img, dict(min_size=4, max_size=16, shift=4, lam=lam), modes=(1, 1, 1, 1))
    _encode_parity(ctx, img, dict(min_size=4, max_size=16, shift=2, lam=lam), modes=(1, 1, 1, 1),
                   adaptive=True, residual_adaptive=True)


def test_forced_border_splits_encode_parity(ctx):
    imgs, _ = fixture_images()
    for name in ("mixed_129x127", "mixed_250x250"):
        _encode_parity(ctx, imgs[name], dict(min_size=4, max_size=32, shift=4, t_rms=8.0))
        _encode_parity(ctx, imgs[name], dict(min_size=4, max_size=16, shift=2, lam=200.0),
                       modes=(1, 1, 1, 0), adaptive=True)


def test_ifs_bytes_identical_through_gpu_encode(ctx):
    # Threshold walk -> .ifs writer: identical bytes from the GPU provider and the oracle.
    img = synthetic.gray(128, 128, 11)
    p = dict(min_size=4, max_size=16, shift=4, t_rms=8.0)
    gh, gl = _encode_parity(ctx, img, p)
    oh, ol, _, _, _ = orc.encode(img, orc.make_params(**p))
    assert mb.ifs_write(gh, gl) == orc.ifs_write(oh, ol)


def test_table_lookup_every_node_matches_oracle(ctx):
    img = synthetic.gray(128, 96, 4)
    p = mb.make_params(min_size=4, max_size=16, shift=2)
    prov = ctx.search_provider(img, p)
    op = orc.make_params(min_size=4, max_size=16, shift=2)
    for size in (4, 8, 16):
        rows, cols = np.meshgrid(np.arange(96 // size) * size, np.arange(128 // size) * size,
                                 indexing="ij")
        o, oev = orc.search_blocks(img, size, 2, op, rows.ravel(), cols.ravel())
        for k, (r, c) in enumerate(zip(rows.ravel(), cols.ravel())):
            out = prov.search(int(r), int(c), size, 2)
            assert out.evals == oev[k]
            cand = out.candidate
            assert cand is not None
            assert (cand.dom_row, cand.dom_col, cand.isometry, cand.qalfa, cand.qbeta) == (
                o[k]["dom_row"], o[k]["dom_col"], o[k]["isometry"], o[k]["qalfa"], o[k]["qbeta"])
            assert cand.rms == o[k]["rms"]
    with pytest.raises(mb.MarsError) as e:
        prov.search(1, 0, 4, 2)
    assert e.value.code == -5
    prov.close()


@pytest.mark.parametrize("entry", mars1_manifest()["fixtures"], ids=lambda e: e["stem"])
def test_gpu_decode_matches_pinned_hash(ctx, entry):
    # crates/mars-codec/tests/ifs.rs:26-107 over all 142 golden streams: 10 iterations.
    hdr, leaves = mb.ifs_parse(mars1_bytes(entry))
    img = ctx.decode(hdr, leaves, 10)
    assert hashlib.sha256(orc.pgm_bytes(img)).hexdigest() == entry["decode_iterative_sha256"]


def test_gpu_decode_modes_0_1_2_match_oracle(ctx):
    img = synthetic.gray(128, 128, 2)
    hdr, leaves, _, _ = ctx.encode(img, mb.make_params(min_size=4, max_size=16, shift=4,
                                                       lam=100.0), allowed_modes=(1, 1, 1, 0))
    assert set(np.unique(leaves["mode"])) <= {0, 1, 2}
    oh = orc.Header(*[getattr(hdr, f) for f, _ in orc.Header._fields_])
    for iters in (1, 3, 12):
        assert np.array_equal(ctx.decode(hdr, leaves, iters), orc.decode(oh, leaves, iters))


@pytest.mark.parametrize("qstep", [0.0, 3.5, 17.123456789])
def test_gpu_decode_mode_3_matches_oracle(ctx, qstep):
    # decode_leaf with the DCT residual (ifs.rs:441-456): the residual is rebuilt on the host
    # and added in the gather.
    img = synthetic.gray(160, 128, 6)
    hdr, leaves, res, _ = ctx.encode(img, mb.make_params(min_size=4, max_size=16, shift=2,
                                                         lam=20.0), allowed_modes=(1, 1, 1, 1),
                                     residual_qstep=qstep)
    assert 3 in set(leaves["mode"].tolist()) and len(res) > 0
    oh = orc.Header(*[getattr(hdr, f) for f, _ in orc.Header._fields_])
    for iters in (1, 2, 10):
        assert np.array_equal(ctx.decode(hdr, leaves, iters, res),
                              orc.decode(oh, leaves, iters, res))


def test_invalid_arguments_are_rejected(ctx):
    img = synthetic.gray(64, 64, 1)
    with pytest.raises(mb.MarsError) as e:
        ctx.search_blocks(img, 4, 3, mb.make_params(shift=3), [0], [0])
    assert e.value.code == -8
    with pytest.raises(mb.MarsError) as e:
        ctx.search_blocks(img, 4, 2, mb.make_params(), [62], [0])
    assert e.value.code == -1
    with pytest.raises(mb.MarsError):
        ctx.encode(img, mb.make_params(lam=float("nan")))
    with pytest.raises(mb.MarsError) as e:
        ctx.encode(img, mb.make_params(lam=10.0), residual_qstep=0.5)
    assert e.value.code == -1
    bad = np.zeros(1, dtype=mb.LEAF_DTYPE)
    bad[0] = (0, 0, 8, 2, 3, 10, 0, 60, 0, 0, 0)  # domain runs past a 64x64 plane
    with pytest.raises(mb.MarsError):
        ctx.decode(mb.Header(4, 7, 4, 16, 4, 64, 64, 32), bad, 2)


@pytest.mark.parametrize("shift", [2, 4, 8, 16])
def test_tensor_core_path_equals_cuda_core_path(ctx, shift):
    # Same blocks through the tcgen05 correlation and through the CUDA-core correlation:
    # identical records, and identical to the oracle.
    img = synthetic.gray(288, 224, 9)
    simt = mb.Context(0)
    simt.set_search_path("simt")
    boxes = mb.Context(0)
    boxes.set_search_path("boxes")  # tensor cores, A stages loaded as per-phase 2-D boxes
    fold = mb.Context(0)
    fold.set_search_path("fold")  # tensor cores, pixels with the 2x2 box folded into K
    try:
        for size in (4, 8, 16, 32, 64):
            if 2 * size > 224:
                continue
            p = mb.make_params(shift=shift)
            a, aev = ctx.search_grid(img, size, shift, p)  # split digits at sizes 16..64
            b, bev = simt.search_grid(img, size, shift, p)
            c, _ = boxes.search_grid(img, size, shift, p)
            d, _ = fold.search_grid(img, size, shift, p)
            assert np.array_equal(aev, bev)
            assert a.tobytes() == b.tobytes(), (size, shift)
            assert c.tobytes() == a.tobytes(), (size, shift)
            assert d.tobytes() == a.tobytes(), (size, shift)
    finally:
        simt.close()
        boxes.close()
        fold.close()
    o, _ = orc.search_grid(img, 8, shift, orc.make_params(shift=shift))
    a, _ = ctx.search_grid(img, 8, shift, mb.make_params(shift=shift))
    assert a.tobytes() == o.tobytes()


def test_device_entry_rejects_blocks_outside_the_plane(ctx):
    # Out-of-plane origins handed to the device-pointer entry are never read and come
    # back invalid, on both correlation paths.
    import torch
    img = synthetic.gray(128, 128, 3)
    d_img = torch.from_numpy(img).cuda()
    rows = torch.tensor([0, 124, 120], dtype=torch.int32, device="cuda")
    cols = torch.tensor([0, 0, 124], dtype=torch.int32, device="cuda")
    out = torch.zeros((3, 80), dtype=torch.uint8, device="cuda")
    p = mb.make_params(shift=2)
    torch.cuda.synchronize()
    mb.check(mb.lib().mars_search_blocks_device(ctx.handle, d_img.data_ptr(), 128, 128, 8, 2,
                                                mb.C.byref(p), rows.data_ptr(), cols.data_ptr(),
                                                3, out.data_ptr()))
    torch.cuda.synchronize()
    rec = out.cpu().numpy().view(mb.CANDIDATE_DTYPE).ravel()
    assert rec[0]["valid"] == 1 and rec[1]["valid"] == 0 and rec[2]["valid"] == 0
    o, _ = orc.search(img, 0, 0, 8, 2, orc.make_params(shift=2))
    assert rec[0].tobytes() == o[0].tobytes()


@pytest.mark.parametrize("threads", ["1", "3", "64"])
def test_host_walk_threads_do_not_change_the_encode(ctx, monkeypatch, threads):
    # The walks run their independent subtrees on a pool of host threads; any pool size
    # gives the sequential walk's leaves, residuals and eval counts.
    img = synthetic.gray(200, 168, 12)
    p = mb.make_params(min_size=4, max_size=16, shift=2, lam=200.0)
    monkeypatch.setenv("MARS_HOST_THREADS", "1")
    ref = ctx.encode(img, p, allowed_modes=(1, 1, 1, 1))
    monkeypatch.setenv("MARS_HOST_THREADS", threads)
    got = ctx.encode(img, p, allowed_modes=(1, 1, 1, 1))
    assert np.array_equal(got[1], ref[1]) and np.array_equal(got[2], ref[2])
    assert (got[3].search_evals, got[3].warmup_evals) == (ref[3].search_evals, ref[3].warmup_evals)
    _encode_parity(ctx, img, dict(min_size=4, max_size=16, shift=2, lam=200.0), modes=(1, 1, 1, 1))


def test_uneven_batch_encodes(ctx):
    # The uneven-batch workload in miniature: planes of the batch's side set, exhaustive
    # search 32..4 at stride 2, lambda 200, encoded one after another on one context.
    sides = [s for s in synthetic.batch_sides(64, 5) if s <= 256][:3]
    assert len(set(sides)) >= 2
    for i, s in enumerate(sides):
        _encode_parity(ctx, synthetic.gray(s, s, 100 + i),
                       dict(min_size=4, max_size=32, shift=2, lam=200.0))


def test_large_plane_sampled_nodes(ctx):
    # A 2048x2048 plane of the generator: a scattered sample of nodes of every size checked
    # against the oracle's search of those nodes (its exhaustive search of one 32x32 node
    # at this size takes seconds, so the sample thins out with the size).
    img = synthetic.gray(2048, 2048, 99)
    prov = ctx.search_provider(img, mb.make_params(min_size=4, max_size=32, shift=2))
    p = orc.make_params(min_size=4, max_size=32, shift=2)
    rng = np.random.default_rng(1)
    for size, n in ((4, 64), (8, 16), (16, 4), (32, 2)):
        rows = (rng.integers(0, 2048 // size, n) * size).astype(np.uint32)
        cols = (rng.integers(0, 2048 // size, n) * size).astype(np.uint32)
        g, gev = prov.search_many(rows, cols, size, 2)
        o, oev = orc.search_blocks(img, size, 2, p, rows, cols)
        assert np.array_equal(gev, oev) and g.tobytes() == o.tobytes(), size
    prov.close()


@pytest.mark.parametrize("path", ["auto", "simt"])
def test_out_of_plane_blocks_stay_invalid_next_to_black_domains(ctx, path):
    # A black region gives domains with s1 = 0, whose pruning threshold does not depend on
    # the range's brightness; an out-of-plane origin must still come back invalid.
    import torch
    img = synthetic.gray(128, 128, 4)
    img[:48, :48] = 0
    d_img = torch.from_numpy(img).cuda()
    # Origins 1 and 2 leave the plane for every block size (126 + 4 > 128).
    rows = torch.tensor([64, 126, 125, 0], dtype=torch.int32, device="cuda")
    cols = torch.tensor([64, 0, 126, 0], dtype=torch.int32, device="cuda")
    out = torch.zeros((4, 80), dtype=torch.uint8, device="cuda")
    p = mb.make_params(shift=2)
    ctx.set_search_path(path)
    try:
        for size in (4, 8, 16):
            torch.cuda.synchronize()
            mb.check(mb.lib().mars_search_blocks_device(ctx.handle, d_img.data_ptr(), 128, 128,
                                                        size, 2, mb.C.byref(p), rows.data_ptr(),
                                                        cols.data_ptr(), 4, out.data_ptr()))
            torch.cuda.synchronize()
            rec = out.cpu().numpy().view(mb.CANDIDATE_DTYPE).ravel()
            assert rec[1]["valid"] == 0 and rec[2]["valid"] == 0
            for i in (0, 3):
                o, _ = orc.search(img, int(rows[i]), int(cols[i]), size, 2, orc.make_params(shift=2))
                assert rec[i].tobytes() == o[0].tobytes()
    finally:
        ctx.set_search_path("auto")
