"""Planned encodes with both walks on the device -- the warm-up walk (walk, encode.rs:1330-1435,
t_rms = 8 for build_rate_snapshot, encode.rs:1139-1169) over the plan's candidates, the
pricing of every node and the RD walk's leaf-versus-split decisions (walk_rd / split_rd,
encode.rs:1865-2027) -- against the oracle, bit-exact: header, leaves in walk order, mode-3
levels and both eval counters.  Also: the plain walk (no lambda), zero_threshold, residual
steps, planes with forced splits, min_size 2 and max_size 64, trees the device walk cannot
serve (pixel leaves: the host walk takes over), concurrent encodes on one plan, and the same
encodes with the walks pinned to the host (MARS_PLAN_WALK=host) in a child process."""
import os
import subprocess
import sys

import numpy as np
import pytest

import mars_b200 as mb
from mars_b200 import synthetic
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def smooth(w, h, seed):
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:h, 0:w].astype(float)
    img = (128 + 60 * np.sin(x / 37.0 + seed) * np.cos(y / 29.0) + 20 * np.sin((x + y) / 11.0)
           + rng.normal(0, 1.5, (h, w)))
    return np.clip(img, 0, 255).astype(np.uint8)


# (plane, params, allowed_modes, extra planned-encode options)
CASES = [
    (("gray", 128, 128, 71), dict(min_size=4, max_size=32, shift=2, lam=200.0), (1, 0, 1, 0), {}),
    (("gray", 136, 104, 72), dict(min_size=4, max_size=16, shift=2, lam=60.0), (1, 1, 1, 1),
     dict(residual_qstep=4.0)),
    (("gray", 160, 120, 73), dict(min_size=4, max_size=32, shift=4, lam=150.0), (0, 0, 0, 1), {}),
    (("gray", 200, 136, 74), dict(min_size=4, max_size=32, shift=2, lam=300.0), (1, 1, 1, 1),
     dict(residual_adaptive=True)),
    (("gray", 96, 80, 75), dict(min_size=2, max_size=16, shift=2, lam=20.0), (1, 1, 1, 1), {}),
    (("smooth", 192, 144, 76), dict(min_size=8, max_size=64, shift=2, lam=800.0), (1, 1, 1, 1),
     {}),
    (("gray", 112, 96, 77), dict(min_size=4, max_size=16, shift=2), (1, 0, 1, 0), {}),
    (("gray", 112, 96, 78), dict(min_size=4, max_size=16, shift=2, t_rms=12.0,
                                 zero_threshold=2), (1, 0, 1, 0), {}),
    (("gray", 96, 88, 79), dict(min_size=4, max_size=16, shift=2, lam=100.0, zero_threshold=3),
     (1, 1, 1, 1), {}),
]


def plane(spec):
    kind, w, h, seed = spec
    return synthetic.gray(w, h, seed) if kind == "gray" else smooth(w, h, seed)


@pytest.fixture(scope="module")
def ctx():
    c = mb.Context(0)
    yield c
    c.close()


def _oracle(img, kw, modes, extra):
    return orc.encode(img, orc.make_params(**kw), allowed_modes=modes, **extra)


def _same(got, want):
    gh, gl, gr, gc = got
    oh, ol, orr, osev, owev = want
    assert bytes(gh) == bytes(oh)
    assert gl.tobytes() == ol.tobytes()
    assert gr.tobytes() == orr.tobytes()
    assert (gc.search_evals, gc.warmup_evals) == (osev, owev)


@pytest.mark.parametrize("case", range(len(CASES)))
def test_planned_device_walks_match_oracle(ctx, case):
    spec, kw, modes, extra = CASES[case]
    img = plane(spec)
    plan = ctx.search_plan(img.shape[1], img.shape[0], mb.make_params(**kw))
    try:
        got = plan.encode(img, allowed_modes=modes, **extra)
        again = plan.encode(img, allowed_modes=modes, **extra)  # buffers reused
    finally:
        plan.close()
    _same(got, _oracle(img, kw, modes, extra))
    assert got[1].tobytes() == again[1].tobytes() and got[2].tobytes() == again[2].tobytes()


def test_trees_with_pixel_leaves_fall_back_to_the_host_walk(ctx):
    # A 66-wide plane at min_size 1: the edge columns split down to single pixels, which
    # the plan does not search, so this plan keeps the host walk; the encode still matches.
    img = synthetic.gray(66, 40, 80)
    kw = dict(min_size=1, max_size=16, shift=2, lam=200.0)
    plan = ctx.search_plan(66, 40, mb.make_params(**kw))
    try:
        got = plan.encode(img, allowed_modes=(1, 0, 1, 0))
    finally:
        plan.close()
    _same(got, _oracle(img, kw, (1, 0, 1, 0), {}))


def test_concurrent_encodes_share_a_plan(ctx):
    kw = dict(min_size=4, max_size=32, shift=2, lam=200.0)
    imgs = [synthetic.gray(128, 96, 90 + i) for i in range(6)]
    for modes in ((1, 0, 1, 0), (1, 1, 1, 1)):
        many = ctx.encode_many(imgs, mb.make_params(**kw), workers=3, allowed_modes=modes)
        for im, got in zip(imgs, many):
            _same(got, _oracle(im, kw, modes, {}))


_CHILD = r"""
import sys
sys.path.insert(0, %r)
import mars_b200 as mb
from tests.test_gpu_plan_walk import CASES, plane
spec, kw, modes, extra = CASES[%d]
img = plane(spec)
with mb.Context(0) as c:
    plan = c.search_plan(img.shape[1], img.shape[0], mb.make_params(**kw))
    hd, lv, rs, ct = plan.encode(img, allowed_modes=modes, **extra)
    plan.close()
sys.stdout.buffer.write(bytes(hd) + lv.tobytes() + rs.tobytes() +
                        bytes(str((ct.search_evals, ct.warmup_evals)), "ascii"))
"""


@pytest.mark.parametrize("case", [1, 5, 6])
def test_device_walks_match_host_walks(case):
    out = {}
    for where in ("device", "host"):
        env = dict(os.environ)
        env.pop("MARS_PLAN_WALK", None)
        if where == "host":
            env["MARS_PLAN_WALK"] = "host"
        res = subprocess.run([sys.executable, "-c", _CHILD % (ROOT, case)], env=env, cwd=ROOT,
                             capture_output=True, timeout=300)
        assert res.returncode == 0, res.stderr.decode()[-2000:]
        out[where] = res.stdout
    assert out["device"] == out["host"]
