"""The .mars v0 container and its rANS entropy coder (host code, no GPU).

Pinned by the reference's own SHA-256s of encoder output
(crates/mars-codec/tests/search_provider.rs:180-227) -- the two cases that need no mode 3 --
and by the unit tests of crates/mars-entropy/src/lib.rs:366-465 and
crates/mars-codec/src/mars_format.rs:764-905, restated.  Leaves come from the CPU oracle's
encode, so these run without a GPU; the GPU encode path is pinned to the same bytes in
test_gpu_mars_format.py.
"""
import hashlib

import numpy as np
import pytest

import mars_b200 as mb
from oracle import oracle as orc
from tests.golden_data import provider_pattern_16

# (lambda, allowed_modes, residual step, .mars length, search evals, SHA-256), from
# search_provider.rs:43-66 (cases 1 and 4) and :180-227.
PINNED = [
    (None, (1, 0, 1, 0), mb.LEGACY_QSTEP, 53, 608,
     "bb480414035f577917542c7f972cb302f904cecbc79449568d05ad74345e98d8"),
    (50.0, (1, 0, 1, 0), 17.123456789, 53, 1184,
     "44fd4f749006cddd0054b817ba5afd630f356bfa6c18f5b68473e4a300c3885f"),
]


def _mb_header(hdr):
    return mb.Header(*[getattr(hdr, f) for f, _ in mb.Header._fields_])


def _encode(img, **kw):
    modes = kw.pop("modes", (1, 0, 1, 0))
    p = orc.make_params(**kw)
    hdr, leaves, sev, _ = orc.encode(img, p, allowed_modes=modes)
    return _mb_header(hdr), leaves, sev


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


@pytest.mark.parametrize("case", PINNED, ids=["threshold", "rd50_modes02_qstep"])
def test_pinned_pre_provider_streams(case):
    lam, modes, qstep, length, evals, digest = case
    hdr, leaves, sev = _encode(provider_pattern_16(), min_size=4, max_size=8, shift=4, lam=lam,
                               modes=modes)
    assert sev == evals
    data = mb.format_write(hdr, leaves, qstep)
    assert len(data) == length
    assert hashlib.sha256(data).hexdigest() == digest
    h2, q2, l2 = mb.format_read(data)
    assert [getattr(h2, f) for f, _ in mb.Header._fields_] == \
        [getattr(hdr, f) for f, _ in mb.Header._fields_]
    assert q2 == float(np.float32(qstep))
    assert np.array_equal(l2, leaves)


def test_qstep_from_lambda():
    # quant.rs:36-52: sqrt(lambda) * sqrt(6 / ln 2), clamped to [1, 65535], binary32.
    assert mb.qstep_from_lambda(0.0) == 1.0
    assert mb.qstep_from_lambda(1e30) == 65535.0
    assert mb.qstep_from_lambda(200.0) == float(np.float32(np.sqrt(200.0) * np.sqrt(6 / np.log(2))))


def test_round_trips_a_real_encode():
    hdr, leaves, _ = _encode(_ramp_image(64, 48), min_size=4, max_size=16, shift=4)
    h2, _, l2 = mb.format_read(mb.format_write(hdr, leaves))
    assert (h2.width, h2.height, h2.min_size, h2.max_size) == (64, 48, 4, 16)
    assert np.array_equal(np.sort(l2, order=["row", "col", "size"]),
                          np.sort(leaves, order=["row", "col", "size"]))


def test_every_mode_the_rd_search_picks_round_trips():
    hdr, leaves, _ = _encode(_textured_gradient(96, 96), min_size=4, max_size=16, shift=4,
                             lam=40.0, modes=(1, 1, 1, 0))
    assert len(set(leaves["mode"].tolist())) > 1
    _, _, l2 = mb.format_read(mb.format_write(hdr, leaves))
    assert np.array_equal(l2, leaves)


def test_compresses_smaller_than_the_raw_ifs_bitstream():
    hdr, leaves, _ = _encode(_ramp_image(128, 96), min_size=4, max_size=16, shift=4)
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
    hdr, leaves, _ = _encode(_ramp_image(32, 32), min_size=4, max_size=16, shift=4)
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
    hdr, leaves, _ = _encode(_ramp_image(64, 64), min_size=4, max_size=16, shift=4)
    data = mb.format_write(hdr, leaves)
    rng = np.random.default_rng(0)
    outcomes = set()
    for _ in range(300):
        b = bytearray(data)
        for _ in range(int(rng.integers(1, 4))):
            b[int(rng.integers(29, len(b)))] = int(rng.integers(0, 256))
        try:
            _, _, l2 = mb.format_read(bytes(b))
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
    hdr, leaves, _ = _encode(_ramp_image(32, 32), min_size=4, max_size=16, shift=4)
    with pytest.raises(mb.MarsError, match="same position"):
        mb.format_write(hdr, np.concatenate([leaves, leaves[:1]]))
    with pytest.raises(mb.MarsError, match="missing"):
        mb.format_write(hdr, leaves[1:])
    with pytest.raises(mb.MarsError, match="qstep"):
        mb.format_write(hdr, leaves, 0.25)
    m3 = leaves.copy()
    m3["mode"][0] = 3
    with pytest.raises(mb.MarsError) as e:
        mb.format_write(hdr, m3)
    assert e.value.code == -8


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
