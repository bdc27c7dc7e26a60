"""The pinned encmars stream of crates/mars-cli/tests/cli_a_gate.rs:50-70, 223-252: a
128x128 gradient 100 + (r + c) % 5, encoded with --lambda 200 --modes 0,1,2,3 --t-rms 0 and
the CLI defaults (sizes 4..16, stride 4, bits 4/7, max_alfa 1), written as the MARC
container of one gray .mars stream (wrap_gray_stream, color.rs:382-384).  The oracle's
encode reproduces the reference's SHA-256; with adaptive density the stream must differ."""
import hashlib

import numpy as np
import pytest

import mars_b200 as mb
from mars_b200 import color
from oracle import oracle as orc

PINNED = "55ccaacf9b9c0e952673992404cfdf8ebb21e8503ae3d45a67b4e82a5eed3544"


def gradient(size=128):
    r, c = np.mgrid[0:size, 0:size]
    return (100 + (r + c) % 5).astype(np.uint8)


def _marc(h, l, res):
    data = mb.format_write(mb.Header(*[getattr(h, f) for f, _ in h._fields_]), l, res)
    return color.write_container(color.MODE_GRAY, [data])


def test_oracle_reproduces_the_pinned_default_stream():
    p = orc.make_params(min_size=4, max_size=16, shift=4, lam=200.0, t_rms=0.0)
    off = _marc(*orc.encode(gradient(), p, allowed_modes=(1, 1, 1, 1))[:3])
    assert hashlib.sha256(off).hexdigest() == PINNED
    on = _marc(*orc.encode(gradient(), p, allowed_modes=(1, 1, 1, 1), adaptive_density=True)[:3])
    assert hashlib.sha256(on).hexdigest() != PINNED


@pytest.mark.gpu
def test_gpu_encoder_reproduces_the_pinned_default_stream():
    with mb.Context(0) as ctx:
        params = color.ColorEncodeParams(
            mb.make_params(min_size=4, max_size=16, shift=4, lam=200.0, t_rms=0.0),
            mb.make_params(min_size=4, max_size=16, shift=4, lam=200.0, t_rms=0.0))
        data, _ = color.encode_color(ctx, gradient(), params)
        assert hashlib.sha256(data).hexdigest() == PINNED
        on, _ = color.encode_color(ctx, gradient(), color.ColorEncodeParams(
            params.y, params.chroma, adaptive_density=True))
        assert hashlib.sha256(on).hexdigest() != PINNED
