"""The decode-side callers beside decode_iterative in the oracle and the host library:
decode_until_stable (ifs.rs:321-353) and zoom_leaves (ifs.rs:356-392).  zoom_leaves is
host arithmetic, so the library's and the oracle's are compared here on the CPU."""
import numpy as np
import pytest

import mars_b200 as mb
from mars_b200 import synthetic
from oracle import oracle as orc


def _hdr(w, h):
    return orc.Header(4, 7, 4, 32, 2, w, h, 32)


def test_until_stable_matches_the_fixed_count_decode():
    leaves = synthetic.quadtree_leaves(96, 64, 3)
    hdr = _hdr(96, 64)
    img, used = orc.decode_until_stable(hdr, leaves, 0, 40)
    assert 1 <= used <= 40
    assert np.array_equal(img, orc.decode(hdr, leaves, used))
    img2, used2 = orc.decode_until_stable(hdr, leaves, 255, 40)
    assert used2 == 1 and np.array_equal(img2, orc.decode(hdr, leaves, 1))
    # Larger thresholds never need more steps.
    steps = [orc.decode_until_stable(hdr, leaves, t, 60)[1] for t in (0, 1, 2, 4, 8)]
    assert steps == sorted(steps, reverse=True)


@pytest.mark.parametrize("factor", [1.0, 2.0, 0.5, 1.5, 3.0])
def test_zoom_leaves_library_equals_oracle(factor):
    leaves = synthetic.quadtree_leaves(128, 96, 5)
    leaves["qgx"] = np.where(leaves["mode"] == 1, leaves["qgx"], 0)
    leaves["mode"][::7] = np.where(leaves["mode"][::7] == 2, 3, leaves["mode"][::7])
    oh = _hdr(128, 96)
    h1, l1 = orc.zoom_leaves(oh, leaves, factor)
    h2, l2 = mb.zoom_leaves(mb.Header(*[getattr(oh, f) for f, _ in oh._fields_]), leaves, factor)
    assert bytes(h1) == bytes(h2) and l1.tobytes() == l2.tobytes()
    assert (h1.width, h1.height) == (round(128 * factor), round(96 * factor))
    if factor == 1.0:
        assert l1.tobytes() == leaves.tobytes()
    else:
        assert not (l1["mode"] == 3).any()


def test_zoom_half_away_from_zero_and_gradients():
    one = np.zeros(1, dtype=orc.LEAF_DTYPE)
    one[0] = (5, 3, 4, 1, 0, 60, 0, 0, 0, -3, 5)  # mode 1, qgx -3, qgy 5
    h, z = orc.zoom_leaves(_hdr(8, 8), one, 0.5)
    # 5 * 0.5 = 2.5 -> 3, 3 * 0.5 = 1.5 -> 2; -3 / 0.5 = -6, 5 / 0.5 = 10.
    assert (z["row"][0], z["col"][0], z["size"][0], z["qgx"][0], z["qgy"][0]) == (3, 2, 2, -6, 10)
    assert (h.width, h.height) == (4, 4)
    with pytest.raises(mb.MarsError):
        mb.zoom_leaves(mb.Header(4, 7, 4, 32, 2, 8, 8, 32), one, 0.0)
