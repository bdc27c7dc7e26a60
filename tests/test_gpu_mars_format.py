"""The GPU encode path end to end against the reference's pinned .mars streams
(crates/mars-codec/tests/search_provider.rs:180-227): the library's search provider, the
host walks, mode-3 residuals and the rANS container give the reference's exact bytes, and
the stream decodes on the GPU to the oracle's image."""
import hashlib

import numpy as np
import pytest

import mars_b200 as mb
from mars_b200 import synthetic
from oracle import oracle as orc
from tests.golden_data import provider_pattern_16
from tests.test_mars_format import PINNED, PINNED_IDS

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = mb.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("case", PINNED, ids=PINNED_IDS)
def test_pinned_streams_through_the_gpu_encoder(ctx, case):
    lam, modes, opts, length, evals, digest = case
    hdr, leaves, res, cnt = ctx.encode(provider_pattern_16(),
                                       mb.make_params(min_size=4, max_size=8, shift=4, lam=lam),
                                       allowed_modes=modes, **opts)
    assert cnt.search_evals == evals
    assert cnt.warmup_evals == (608 if lam is not None else 0)
    data = mb.format_write(hdr, leaves, res)
    assert len(data) == length
    assert hashlib.sha256(data).hexdigest() == digest
    h2, l2, r2 = mb.format_read(data)
    oh = orc.Header(*[getattr(h2, f) for f, _ in orc.Header._fields_])
    assert np.array_equal(ctx.decode(h2, l2, 10, r2), orc.decode(oh, l2, 10, r2))


def test_default_options_stream(ctx):
    # encmars's defaults: every mode, residual step 8, lambda 200, on a synthetic plane.
    img = synthetic.gray(192, 160, 4)
    params = dict(min_size=4, max_size=32, shift=2, lam=200.0)
    hdr, leaves, res, _ = ctx.encode(img, mb.make_params(**params), allowed_modes=(1, 1, 1, 1))
    oh, ol, ores, _, _ = orc.encode(img, orc.make_params(**params), allowed_modes=(1, 1, 1, 1))
    data = mb.format_write(hdr, leaves, res)
    assert data == mb.format_write(mb.Header(*[getattr(oh, f) for f, _ in oh._fields_]), ol, ores)
    h2, l2, r2 = mb.format_read(data)
    assert np.array_equal(l2, leaves) and np.array_equal(r2, res)
