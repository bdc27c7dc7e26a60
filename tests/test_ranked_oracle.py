"""rd_candidates in the oracle's encode (EncodeOptions::rd_candidates, encode.rs:1946-1977),
with the properties the reference's own tests hold (encode.rs:3040-3127): an explicit 1 is
the default, a list wider than one is deterministic and changes nothing when no domain mode
competes, and the CLI's preconditions (encmars.rs:553-566) are refused."""
import numpy as np
import pytest

from mars_b200 import synthetic
from oracle import oracle as orc


def _bytes(h, l, r):
    import mars_b200 as mb
    return mb.format_write(mb.Header(*[getattr(h, f) for f, _ in h._fields_]), l, r)


def test_explicit_one_is_the_default_and_mode0_ignores_the_width():
    img = synthetic.gray(64, 64, 21)
    p = orc.make_params(min_size=4, max_size=16, shift=4, lam=200.0)
    base = orc.encode(img, p, allowed_modes=(1, 0, 1, 1))
    one = orc.encode(img, p, allowed_modes=(1, 0, 1, 1), rd_candidates=1)
    assert _bytes(*base[:3]) == _bytes(*one[:3])
    m0 = orc.encode(img, p, allowed_modes=(1, 0, 0, 0))
    m0w = orc.encode(img, p, allowed_modes=(1, 0, 0, 0), rd_candidates=4)
    assert _bytes(*m0[:3]) == _bytes(*m0w[:3])


def test_wider_lists_are_deterministic_and_count_the_same_evals():
    img = synthetic.gray(64, 64, 22)
    p = orc.make_params(min_size=4, max_size=16, shift=4, lam=200.0)
    one = orc.encode(img, p, allowed_modes=(1, 0, 1, 1))
    a = orc.encode(img, p, allowed_modes=(1, 0, 1, 1), rd_candidates=3)
    b = orc.encode(img, p, allowed_modes=(1, 0, 1, 1), rd_candidates=3)
    assert _bytes(*a[:3]) == _bytes(*b[:3])
    assert (a[3], a[4]) == (one[3], one[4])


def test_preconditions_are_refused():
    img = synthetic.gray(32, 32, 23)
    with pytest.raises(ValueError):
        orc.encode(img, orc.make_params(min_size=4, max_size=16, shift=4), rd_candidates=2)
    with pytest.raises(ValueError):
        orc.encode(img, orc.make_params(min_size=4, max_size=16, shift=4, lam=200.0),
                   rd_candidates=2, method="fisher")


def test_top_k_search_is_sorted_by_rms_then_order():
    img = synthetic.gray(48, 48, 24)
    p = orc.make_params(min_size=4, max_size=16, shift=2)
    for size in (4, 8):
        c1, e1 = orc.search(img, 8, 8, size, 2, p, k=1)
        c5, e5 = orc.search(img, 8, 8, size, 2, p, k=5)
        assert e1 == e5 and c5[0].tobytes() == c1[0].tobytes()
        keys = [(float(c["rms"]), (int(c["dom_row"]) * 1000 + int(c["dom_col"])) * 8 + int(c["isometry"]))
                for c in c5]
        assert keys == sorted(keys)
