"""Cross-checks against the reference's own 1998 C decoder (reference/mars1), built from
its sources into oracle/_ref/ by `make -C oracle ref` when the reference checkout exists.
Skipped where that binary is absent."""
import hashlib
import os
import subprocess
import tempfile

import numpy as np
import pytest

from mars_b200 import synthetic
from oracle import oracle as orc
from tests.golden_data import mars1_bytes, mars1_manifest

DECMARS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle",
                       "_ref", "decmars")
pytestmark = pytest.mark.skipif(not os.path.exists(DECMARS), reason="oracle/_ref/decmars not built")


def decmars(ifs: bytes, iters=10) -> bytes:
    with tempfile.TemporaryDirectory() as d:
        src, dst = os.path.join(d, "i.ifs"), os.path.join(d, "o.pgm")
        open(src, "wb").write(ifs)
        subprocess.run([DECMARS, "-i", "-n", str(iters), src, dst], check=True, cwd=d,
                       stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        return open(dst, "rb").read()


@pytest.mark.parametrize("entry", mars1_manifest()["fixtures"][::7], ids=lambda e: e["stem"])
def test_reference_decoder_reproduces_pinned_hashes(entry):
    out = decmars(mars1_bytes(entry))
    assert hashlib.sha256(out).hexdigest() == entry["decode_iterative_sha256"]


@pytest.mark.parametrize("seed,lam", [(3, None), (4, None)])
def test_oracle_encode_decodes_identically_in_reference_decoder(seed, lam):
    # Our threshold-walk encode, written as .ifs, decoded by the 1998 C decoder and by the
    # oracle's decode_iterative restatement: identical PGM bytes.
    img = synthetic.gray(128, 96, seed)
    hdr, leaves, _, _, _ = orc.encode(img, orc.make_params(min_size=4, max_size=16, shift=4,
                                                           lam=lam))
    data = orc.ifs_write(hdr, leaves)
    ref = decmars(data)
    ours = orc.pgm_bytes(orc.decode(hdr, leaves, 10))
    assert ref == ours
