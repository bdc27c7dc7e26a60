"""The committed 4096x4096 sample (tests/golden/sample_4096.json) against a fresh oracle run
of one of its nodes per block size 4 and 8: the fixture the GPU test reads is the oracle's."""
import json
import os

import numpy as np
import pytest

from mars_b200 import synthetic
from oracle import oracle as orc

SAMPLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sample_4096.json")


@pytest.mark.parametrize("size", [4, 8])
def test_fixture_node_is_the_oracle(size):
    with open(SAMPLE) as f:
        s = json.load(f)
    lv = s["levels"][str(size)]
    img = synthetic.gray(s["side"], s["side"], s["seed"])
    i = len(lv["rows"]) - 1  # the last sampled node
    cands, evals = orc.search_blocks(img, size, s["shift"],
                                     orc.make_params(min_size=4, max_size=32, shift=s["shift"]),
                                     np.array([lv["rows"][i]], np.uint32),
                                     np.array([lv["cols"][i]], np.uint32))
    assert cands[0].tobytes().hex() == lv["records"][i]
    assert int(evals[0]) == lv["evals"][i]
