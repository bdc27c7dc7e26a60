"""Pins the CPU oracle to the reference's own known answers and golden fixtures.

Each test cites the reference test it mirrors (paths relative to the reference root).
"""
import hashlib

import numpy as np
import pytest

from oracle import oracle as orc
from tests.golden_data import fixture_images, mars1_bytes, mars1_manifest, provider_pattern_16


def test_fit_f64_flat128_worked_example():
    # crates/mars-codec/src/encode.rs:2208-2231
    size = 16
    qa, qb, rms = orc.fit_f64(size * size, 128 * 4 * size * size, 512 * 512 * size * size,
                              128 * size * size, 128 * 512 * size * size, 128 * 128 * size * size)
    assert (qa, qb) == (0, 64)
    assert abs(rms - 0.5039370078736174) < 1e-12


def test_best_beta_zero_alfa_override():
    # crates/mars-codec/src/encode.rs:2234-2241
    assert orc.best_beta(128 * 256, 256, 7) == 64


def _xorshift(seed):
    s = seed
    while True:
        s ^= (s << 13) & 0xFFFFFFFFFFFFFFFF
        s ^= s >> 7
        s ^= (s << 17) & 0xFFFFFFFFFFFFFFFF
        yield s


def test_integer_moments_exact_against_naive_f64():
    # crates/mars-codec/src/encode.rs:2182-2205 (fewer blocks; same xorshift seed).  The
    # oracle's search reports the winner's integer moments; recompute them naively in f64
    # from the same pixels.
    rng = _xorshift(0x5EED_C0DE_1234_5678)
    for _ in range(300):
        size = [2, 4, 8, 16][next(rng) % 4]
        rng_bytes = np.array([next(rng) & 0xFF for _ in range(size * size)], dtype=np.uint8)
        dom = np.array([next(rng) & 0xFF for _ in range(4 * size * size)], dtype=np.uint8)
        # image: range block at (0, 0), one domain at (0, 2*size) -> width 4*size, height 2*size
        img = np.zeros((2 * size, 4 * size), dtype=np.uint8)
        img[:size, :size] = rng_bytes.reshape(size, size)
        img[:, 2 * size:] = dom.reshape(2 * size, 2 * size)
        cands, evals = orc.search(img, 0, 0, size, 2 * size, orc.make_params(), k=1)
        assert evals == 2 * 8
        c = cands[0]
        d = img.astype(np.float64)
        dom_px = d[c["dom_row"]:c["dom_row"] + 2 * size, c["dom_col"]:c["dom_col"] + 2 * size]
        mean = (dom_px[0::2, 0::2] + dom_px[1::2, 0::2] + dom_px[0::2, 1::2] + dom_px[1::2, 1::2]) / 4.0
        assert c["s1_x4"] / 4.0 == mean.sum()
        assert c["s2_x16"] / 16.0 == (mean * mean).sum()
        r = d[:size, :size]
        assert c["t0"] == r.sum() and c["t2"] == (r * r).sum()
        # isometry::map applied to the domain sample grid
        k = int(c["isometry"])
        t1 = 0.0
        for u in range(size):
            for v in range(size):
                i, j = {0: (u, v), 1: (size - 1 - v, u), 2: (v, size - 1 - u),
                        3: (size - 1 - u, size - 1 - v), 4: (u, size - 1 - v),
                        5: (size - 1 - u, v), 6: (v, u), 7: (size - 1 - v, size - 1 - u)}[k]
                t1 += r[i, j] * mean[u, v]
        assert c["t1_x4"] / 4.0 == t1


def test_provider_pattern_pinned_evals():
    # crates/mars-codec/tests/search_provider.rs:29-66,180-227: the evals column of
    # pinned_pre_provider_streams (608 threshold; 1184 RD; 864 RD + adaptive density;
    # 1184 RD lambda 50 with modes {0, 2}).  RD evals do not depend on which modes compete.
    img = provider_pattern_16()
    p = dict(min_size=4, max_size=8, shift=4, t_rms=8.0)
    _, _, _, sev, wev = orc.encode(img, orc.make_params(**p))
    assert (sev, wev) == (608, 0)
    _, _, _, sev, wev = orc.encode(img, orc.make_params(lam=2.0, **p), allowed_modes=(1, 1, 1, 1))
    assert (sev, wev) == (1184, 608)
    _, _, _, sev, wev = orc.encode(img, orc.make_params(lam=2.0, **p), allowed_modes=(1, 1, 1, 1),
                                   adaptive_density=True, residual_adaptive=True)
    assert (sev, wev) == (864, 608)
    _, _, _, sev, wev = orc.encode(img, orc.make_params(lam=50.0, **p), allowed_modes=(1, 0, 1, 0),
                                   residual_qstep=17.123456789)
    assert (sev, wev) == (1184, 608)


def test_provider_pattern_recorded_requests():
    # crates/mars-codec/tests/search_provider.rs:114-177: the final RD walk makes 20 searches
    # (4 size-8 parents + 16 size-4 children); every leaf then tiles the 16x16 plane.
    img = provider_pattern_16()
    hdr, leaves, _, sev, _ = orc.encode(img, orc.make_params(min_size=4, max_size=8, shift=4,
                                                             lam=2.0))
    assert sev == 4 * 8 + 16 * 72
    cover = np.zeros((16, 16), dtype=np.int32)
    for l in leaves:
        cover[l["row"]:l["row"] + l["size"], l["col"]:l["col"] + l["size"]] += 1
    assert (cover == 1).all()


@pytest.mark.parametrize("entry", mars1_manifest()["fixtures"], ids=lambda e: e["stem"])
def test_mars1_ifs_parse_write_decode(entry):
    # crates/mars-codec/tests/ifs.rs:26-107 over all 142 entries of fixtures/mars1/manifest.toml
    data = mars1_bytes(entry)
    assert hashlib.sha256(data).hexdigest() == entry["ifs_sha256"]
    hdr, leaves = orc.ifs_parse(data)
    assert (hdr.width, hdr.height) == (entry["width"], entry["height"])
    assert (hdr.min_size, hdr.max_size, hdr.shift) == (entry["min_size"], entry["max_size"],
                                                       entry["shift"])
    assert len(leaves) == entry["transforms"]
    assert int((leaves["qalfa"] == 0).sum()) == entry["zero_alfa_transforms"]
    assert orc.ifs_write(hdr, leaves) == data
    img = orc.decode(hdr, leaves, 10)
    assert hashlib.sha256(orc.pgm_bytes(img)).hexdigest() == entry["decode_iterative_sha256"]


def test_tiny64_walkthrough_table():
    # crates/mars-codec/tests/ifs.rs:58-107
    entry = next(e for e in mars1_manifest()["fixtures"] if e["stem"] == "tiny64__walkthrough__fisher__r8")
    hdr, leaves = orc.ifs_parse(mars1_bytes(entry))
    expected = [(0, 0, 32, 0, 50, 0, 0, 0), (32, 0, 16, 8, 49, 0, 32, 0), (48, 0, 16, 8, 70, 0, 32, 0),
                (32, 16, 16, 8, 49, 0, 32, 0), (48, 16, 16, 8, 70, 0, 32, 0),
                (0, 32, 32, 0, 85, 0, 0, 0), (32, 32, 32, 0, 30, 0, 0, 0)]
    got = [tuple(int(l[k]) for k in ("row", "col", "size", "qalfa", "qbeta", "isometry", "dom_row",
                                     "dom_col")) for l in leaves]
    assert got == expected


def test_fixture_images_match_reference_pins():
    imgs, meta = fixture_images()
    for m in meta:
        a = imgs[m["name"]]
        assert a.shape == (m["height"], m["width"])
        assert hashlib.sha256(a.tobytes()).hexdigest() == m["sha256"]


def test_exhaustive_grid_equals_per_block_search():
    # crates/mars-search/src/lib.rs:824-904 in spirit: the bulk grid search and the
    # single-block search_top_k agree on winner, rms and evals (32x32 xorshift image).
    rng = _xorshift(0x1234_5678_9ABC_DEF0)
    img = np.array([next(rng) & 0xFF for _ in range(32 * 32)], dtype=np.uint8).reshape(32, 32)
    p = orc.make_params()
    for size in (4, 8, 16):
        grid, ev = orc.search_grid(img, size, 4, p, nthreads=2)
        for b, (i, j) in enumerate([(i, j) for i in range(32 // size) for j in range(32 // size)]):
            one, ev1 = orc.search(img, i * size, j * size, size, 4, p)
            assert ev[b] == ev1
            if size == 16:
                assert ev1 == 8
            assert one[0].tobytes() == grid[b].tobytes()


def test_thread_count_identity():
    # crates/mars-codec/tests/parallel_determinism.rs:36-84 (mixed_129x127, min 4, max 32,
    # shift 4, t_rms 8): leaves and evals identical at 1, 2 and 4 threads.
    imgs, _ = fixture_images()
    img = imgs["mixed_129x127"]
    p = orc.make_params(min_size=4, max_size=32, shift=4, t_rms=8.0)
    base = orc.encode(img, p, nthreads=1)
    for nt in (2, 4):
        again = orc.encode(img, p, nthreads=nt)
        assert again[3] == base[3]
        assert again[1].tobytes() == base[1].tobytes()


def test_top_k_prefix_and_winner():
    # crates/mars-codec/src/encode.rs:2989 (top-k prefix/winner invariance)
    imgs, _ = fixture_images()
    img = imgs["zoneplate"][:64, :64]
    p = orc.make_params()
    one, ev1 = orc.search(img, 8, 16, 8, 4, p, k=1)
    many, evk = orc.search(img, 8, 16, 8, 4, p, k=5)
    assert ev1 == evk and one[0].tobytes() == many[0].tobytes()
    assert list(many["rms"]) == sorted(many["rms"])
