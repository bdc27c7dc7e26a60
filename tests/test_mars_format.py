"""The .mars v0 container and its rANS entropy coder (host code, no GPU).

Pinned by the reference's own SHA-256s of encoder output
(crates/mars-codec/tests/search_provider.rs:180-227: all four streams, two of them with mode-3
DCT residuals) and by the unit tests of crates/mars-entropy/src/lib.rs:366-465,
crates/mars-codec/src/mars_format.rs:764-905, dct.rs and quant.rs, restated.  Leaves come
from the CPU oracle's encode, so these run without a GPU; the GPU encode path is pinned to
the same bytes in test_gpu_mars_format.py.
"""
import hashlib

import numpy as np
import pytest

import mars_b200 as mb
from oracle import oracle as orc
from tests.golden_data import provider_pattern_16

# search_provider.rs:43-66 (the four cases) and :180-227 (length, evals, SHA-256): threshold;
# RD lambda 2 with every mode; RD lambda 2 + adaptive density + lambda-adaptive residual step;
# RD lambda 50, modes {0, 2}, fixed step 17.123456789.
PINNED = [
    (None, (1, 1, 1, 1), {}, 53, 608,
     "bb480414035f577917542c7f972cb302f904cecbc79449568d05ad74345e98d8"),
    (2.0, (1, 1, 1, 1), {}, 149, 1184,
     "5069a669a65b6926bc8a597099e0c40c36ac94f038138480226c9b0385b6ae1c"),
    (2.0, (1, 1, 1, 1), dict(adaptive_density=True, residual_adaptive=True), 161, 864,
     "afbb23207c8e98b70a1b23639701a8c02d46bd10e7299c58cebe60d52cee76d8"),
    (50.0, (1, 0, 1, 0), dict(residual_qstep=17.123456789), 53, 1184,
     "44fd4f749006cddd0054b817ba5afd630f356bfa6c18f5b68473e4a300c3885f"),
]
PINNED_IDS = ["threshold", "rd2_all_modes", "rd2_density_adaptive", "rd50_modes02_qstep"]


def _mb_header(hdr):
    return mb.Header(*[getattr(hdr, f) for f, _ in mb.Header._fields_])


def _encode(img, modes=(1, 0, 1, 0), opts=None, **kw):
    hdr, leaves, res, sev, _ = orc.encode(img, orc.make_params(**kw), allowed_modes=modes,
                                          **(opts or {}))
    return _mb_header(hdr), leaves, res, sev


def _ramp_image(w, h):
    # mars_format.rs:740-748
    r, c = np.mgrid[0:h, 0:w]
    return ((r * 7 + c * 13) % 256).astype(np.uint8)


def _textured_gradient(w, h):
    # mars_format.rs:801-814
    r, c = np.mgrid[0:h, 0:w]
    base = r * 255 // max(h, 1)
    texture = ((r // 4) * 13 + (c // 4) * 7) % 32 - 16
    return np.clip(base + texture, 0, 255).astype(np.uint8)


@pytest.mark.parametrize("case", PINNED, ids=PINNED_IDS)
def test_pinned_pre_provider_streams(case):
    lam, modes, opts, length, evals, digest = case
    hdr, leaves, res, sev = _encode(provider_pattern_16(), modes, opts, min_size=4, max_size=8,
                                    shift=4, lam=lam)
    assert sev == evals
    data = mb.format_write(hdr, leaves, res)
    assert len(data) == length
    assert hashlib.sha256(data).hexdigest() == digest
    h2, l2, r2 = mb.format_read(data)
    assert bytes(h2) == bytes(hdr)
    assert np.array_equal(l2, leaves) and np.array_equal(r2, res)


def test_qstep_from_lambda():
    # quant.rs:36-52: sqrt(lambda) * sqrt(6 / ln 2), clamped to [1, 65535], binary32.
    assert mb.qstep_from_lambda(0.0) == 1.0
    assert mb.qstep_from_lambda(1e30) == 65535.0
    assert mb.qstep_from_lambda(200.0) == float(np.float32(np.sqrt(200.0) * np.sqrt(6 / np.log(2))))
    hdr, _, _, _ = _encode(provider_pattern_16(), (1, 1, 1, 1), dict(residual_adaptive=True),
                           min_size=4, max_size=8, shift=4, lam=2.0)
    assert hdr.residual_qstep == mb.qstep_from_lambda(2.0)


def test_round_trips_a_real_encode():
    hdr, leaves, _, _ = _encode(_ramp_image(64, 48), min_size=4, max_size=16, shift=4)
    h2, l2, _ = mb.format_read(mb.format_write(hdr, leaves))
    assert (h2.width, h2.height, h2.min_size, h2.max_size) == (64, 48, 4, 16)
    assert np.array_equal(np.sort(l2, order=["row", "col", "size"]),
                          np.sort(leaves, order=["row", "col", "size"]))


def test_every_mode_the_rd_search_picks_round_trips():
    # mars_format.rs:816-851: a lambda-40 RD encode of the textured gradient uses several
    # modes, mode 3's residual included, and every field round-trips.
    hdr, leaves, res, _ = _encode(_textured_gradient(96, 96), (1, 1, 1, 1), min_size=4,
                                  max_size=16, shift=4, lam=40.0)
    assert len(set(leaves["mode"].tolist())) > 1
    h2, l2, r2 = mb.format_read(mb.format_write(hdr, leaves, res))
    assert np.array_equal(l2, leaves) and np.array_equal(r2, res)


def test_compresses_smaller_than_the_raw_ifs_bitstream():
    hdr, leaves, _, _ = _encode(_ramp_image(128, 96), min_size=4, max_size=16, shift=4)
    assert len(mb.format_write(hdr, leaves)) < len(mb.ifs_write(hdr, leaves))


def _expect(data, text):
    with pytest.raises(mb.MarsError) as e:
        mb.format_read(data)
    assert e.value.code == -7 and text in str(e.value)


def test_rejects_malformed_containers():
    bad = bytearray(29)
    bad[0:4] = b"NOPE"
    _expect(bytes(bad), "bad magic")
    _expect(b"", "truncated")
    _expect(b"MARS", "truncated")
    hdr, leaves, _, _ = _encode(_ramp_image(32, 32), min_size=4, max_size=16, shift=4)
    data = bytearray(mb.format_write(hdr, leaves))
    data[25:29] = (0xFFFFFFFF).to_bytes(4, "little")
    _expect(bytes(data), "section table claims")
    deg = bytearray(29)
    deg[0:4] = b"MARS"
    deg[20:24] = np.float32(8.0).tobytes()
    deg[12], deg[13], deg[11] = 0, 4, 4
    deg[15:17] = (16).to_bytes(2, "little")
    deg[17:19] = (16).to_bytes(2, "little")
    _expect(bytes(deg), "degenerate header")
    v = bytearray(mb.format_write(hdr, leaves))
    v[4] = 1
    _expect(bytes(v), "version")
    q = bytearray(mb.format_write(hdr, leaves))
    q[20:24] = np.float32(0.5).tobytes()
    _expect(bytes(q), "qstep")
    nt = bytearray(mb.format_write(hdr, leaves))
    nt[24] = 2  # the only section is no longer TREE
    _expect(bytes(nt), "TREE section is missing")


def test_corrupted_payloads_never_crash():
    # mars_format::read must reject or decode arbitrary bytes without faulting (the reference
    # fuzzes it, fuzz/fuzz_targets/mars_format_read.rs).
    hdr, leaves, res, _ = _encode(_ramp_image(64, 64), (1, 1, 1, 1), min_size=4, max_size=16,
                                  shift=4, lam=30.0)
    data = mb.format_write(hdr, leaves, res)
    rng = np.random.default_rng(0)
    outcomes = set()
    for _ in range(300):
        b = bytearray(data)
        for _ in range(int(rng.integers(1, 4))):
            b[int(rng.integers(29, len(b)))] = int(rng.integers(0, 256))
        try:
            _, l2, _ = mb.format_read(bytes(b))
            assert ((l2["row"] + l2["size"] <= 64) & (l2["col"] + l2["size"] <= 64)).all()
            outcomes.add("ok")
        except mb.MarsError as e:
            assert e.code in (-7, -8)
            outcomes.add(e.code)
    for cut in range(len(data)):
        try:
            mb.format_read(data[:cut])
        except mb.MarsError:
            pass
    assert outcomes


def test_writer_rejects_bad_leaf_sets():
    hdr, leaves, _, _ = _encode(_ramp_image(32, 32), min_size=4, max_size=16, shift=4)
    with pytest.raises(mb.MarsError, match="same position"):
        mb.format_write(hdr, np.concatenate([leaves, leaves[:1]]))
    with pytest.raises(mb.MarsError, match="missing"):
        mb.format_write(hdr, leaves[1:])
    bad = _mb_header(hdr)
    bad.residual_qstep = 0.25
    with pytest.raises(mb.MarsError, match="qstep"):
        mb.format_write(bad, leaves)
    m3 = leaves.copy()
    k = int(np.flatnonzero(m3["mode"] == 2)[0])
    m3["mode"][k] = 3  # a mode-3 leaf needs size*size residual levels
    with pytest.raises(mb.MarsError, match="residual pool"):
        mb.format_write(hdr, m3)
    n = int(m3["size"][k]) ** 2
    levels = np.arange(n) % 7 - 3
    assert mb.format_read(mb.format_write(hdr, m3, levels))[2].tolist() == levels.tolist()


def test_dct_and_dead_zone_restatements():
    # dct.rs:97-151 and quant.rs:118-152 restated: round trip within 1e-9, DC-only energy
    # for a constant block, requantising a dequantised level is the identity.
    rng = np.random.default_rng(1)
    for size in (2, 4, 8, 16):
        block = rng.random((size, size)) * 255.0
        back = orc.inverse_dct2d(orc.forward_dct2d(block))
        assert np.abs(back - block).max() < 1e-9
    c = orc.forward_dct2d(np.full((8, 8), 100.0))
    assert abs(c[0, 0] - 800.0) < 1e-9 and np.abs(c.ravel()[1:]).max() < 1e-9
    assert orc.dead_zone_quantize(0.0, 4.0, 0.5) == 0
    for _ in range(2000):
        step = max(rng.random() * 25.0, 0.05)
        dz = min(rng.random() / 2.0, 0.49)
        level = int(rng.integers(-63, 64))
        assert orc.dead_zone_quantize(orc.dead_zone_dequantize(level, step, dz), step, dz) == level


# crates/mars-entropy/src/lib.rs:366-465


def test_entropy_round_trips_a_skewed_stream():
    symbols = [1 if i % 7 == 0 else 0 for i in range(2000)]
    data = mb.entropy_encode([(0, 0, 2, s) for s in symbols])
    assert mb.entropy_decode(data, [(0, 0, 2)] * len(symbols)) == symbols
    assert len(data) < 2000 // 8 * 3


def test_entropy_round_trips_multiple_contexts_and_alphabets():
    events = []
    for i in range(500):
        ctx, alphabet = (i % 3, i % 5), 4 + (i % 3) * 10
        events.append((ctx[0], ctx[1], alphabet, i % alphabet))
    data = mb.entropy_encode(events)
    assert mb.entropy_decode(data, [e[:3] for e in events]) == [e[3] for e in events]


def test_entropy_single_symbol_alphabet_is_rejected():
    with pytest.raises(mb.MarsError):
        mb.entropy_encode([(0, 0, 1, 0)])
    with pytest.raises(mb.MarsError):
        mb.entropy_encode([(0, 0, 4, 4)])  # symbol outside its alphabet


def test_entropy_large_alphabets_and_rescaling():
    rng = np.random.default_rng(3)
    events = [(5, 1, 4097, int(s)) for s in rng.integers(0, 4097, 5000)]
    events += [(2, 2, 3, int(s)) for s in rng.integers(0, 3, 30000)]  # crosses 2^16 totals
    data = mb.entropy_encode(events)
    assert mb.entropy_decode(data, [e[:3] for e in events]) == [e[3] for e in events]
    assert mb.entropy_encode([]) == b""
    assert mb.entropy_decode(b"", []) == []
    with pytest.raises(mb.MarsError):
        mb.entropy_decode(b"\x01\x00\x00\x00\x00\x00\x00\x00", [(0, 0, 2)])  # trailing zero word
