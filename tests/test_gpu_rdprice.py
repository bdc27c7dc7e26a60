"""RD pricing on the device (best_mode_leaf, encode.rs:1536-1714, for every node walk_rd can
visit, one warp per node) against the oracle's host walk, bit-exact: whole RD encodes --
header, leaves, mode-3 residual levels and eval counters -- across node sizes 2..64, every
mode mix, ranked candidate lists, adaptive density and planes with forced splits; the same
encodes priced by the host walk (MARS_PRICING=host, the same price_node as a team of one
lane) in a child process; and modes 0-2 encodes (host-priced by default) pinned to the
device."""
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
    """A smooth plane with light noise, on which 32x32 leaves win at a high lambda."""
    rng = np.random.default_rng(seed)
    y, x = np.mgrid[0:h, 0:w].astype(float)
    img = (128 + 60 * np.sin(x / 37.0 + seed) * np.cos(y / 29.0) + 20 * np.sin((x + y) / 11.0)
           + rng.normal(0, 1.5, (h, w)))
    return np.clip(img, 0, 255).astype(np.uint8)


# (plane, params, allowed_modes, extra options, a mode-3 leaf expected)
CASES = [
    (("gray", 136, 104, 61), dict(min_size=2, max_size=16, shift=2, lam=20.0), (1, 1, 1, 1),
     dict(residual_qstep=4.0), True),
    (("gray", 192, 144, 62), dict(min_size=8, max_size=64, shift=2, lam=10.0), (1, 1, 1, 1),
     {}, True),
    (("gray", 160, 120, 63), dict(min_size=4, max_size=32, shift=4, lam=150.0), (0, 0, 0, 1),
     {}, True),
    (("gray", 128, 96, 64), dict(min_size=4, max_size=16, shift=2, lam=200.0), (1, 0, 1, 1),
     dict(rd_candidates=4), False),
    (("gray", 144, 112, 65), dict(min_size=4, max_size=32, shift=2, lam=120.0), (1, 1, 1, 1),
     dict(adaptive_density=True), False),
    (("gray", 96, 80, 66), dict(min_size=4, max_size=16, shift=2, lam=250.0), (1, 1, 1, 1),
     dict(residual_adaptive=True), False),
    (("smooth", 192, 144, 68), dict(min_size=8, max_size=64, shift=2, lam=800.0), (1, 1, 1, 1),
     {}, False),
]


def plane(spec):
    kind, w, h, seed = spec
    return synthetic.gray(w, h, seed) if kind == "gray" else smooth(w, h, seed)


@pytest.fixture(scope="module")
def ctx():
    c = mb.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("case", range(len(CASES)))
def test_device_pricing_matches_oracle(ctx, case):
    spec, kw, modes, extra, want3 = CASES[case]
    img = plane(spec)
    gh, gl, gr, gc = ctx.encode(img, mb.make_params(**kw), allowed_modes=modes, **extra)
    oh, ol, orr, osev, owev = orc.encode(img, orc.make_params(**kw), allowed_modes=modes, **extra)
    assert bytes(gh) == bytes(oh)
    assert gl.tobytes() == ol.tobytes()
    assert gr.tobytes() == orr.tobytes()
    assert (gc.search_evals, gc.warmup_evals) == (osev, owev)
    if want3:
        assert (gl["mode"] == 3).any(), "the case should exercise the residual mode"
    if spec[0] == "smooth":
        assert (gl["size"] == 32).any(), "the case should keep 32x32 leaves"


_CHILD = r"""
import sys
sys.path.insert(0, %r)
import mars_b200 as mb
from tests.test_gpu_rdprice import CASES, plane
spec, kw, modes, extra, _ = CASES[%d]
with mb.Context(0) as c:
    hd, lv, rs, ct = c.encode(plane(spec), mb.make_params(**kw), allowed_modes=modes, **extra)
sys.stdout.buffer.write(bytes(hd) + lv.tobytes() + rs.tobytes())
"""


@pytest.mark.parametrize("case", [0, 1, 3, 6])
def test_device_pricing_matches_host_pricing(case):
    out = {}
    for where in ("device", "host"):
        env = dict(os.environ, MARS_PRICING=where)
        res = subprocess.run([sys.executable, "-c", _CHILD % (ROOT, case)], env=env, cwd=ROOT,
                             capture_output=True, timeout=300)
        assert res.returncode == 0, res.stderr.decode()[-2000:]
        out[where] = res.stdout
    assert out["device"] == out["host"]


_CHILD_MODES = r"""
import sys
sys.path.insert(0, %r)
import mars_b200 as mb
from oracle import oracle as orc
from mars_b200 import synthetic
img = synthetic.gray(144, 120, 69)
kw = dict(min_size=4, max_size=32, shift=2, lam=150.0)
for modes in ((1, 0, 1, 0), (1, 1, 1, 0), (0, 1, 0, 0)):
    with mb.Context(0) as c:
        gh, gl, gr, gc = c.encode(img, mb.make_params(**kw), allowed_modes=modes)
    oh, ol, orr, osev, owev = orc.encode(img, orc.make_params(**kw), allowed_modes=modes)
    assert bytes(gh) == bytes(oh) and gl.tobytes() == ol.tobytes(), modes
    assert (gc.search_evals, gc.warmup_evals) == (osev, owev), modes
print("ok")
"""


def test_modes_without_residual_priced_on_device():
    env = dict(os.environ, MARS_PRICING="device")
    res = subprocess.run([sys.executable, "-c", _CHILD_MODES % ROOT], env=env, cwd=ROOT,
                         capture_output=True, timeout=300)
    assert res.returncode == 0, res.stderr.decode()[-2000:]
    assert res.stdout.strip().endswith(b"ok")


def test_planned_encode_prices_on_device(ctx):
    img = synthetic.gray(128, 128, 67)
    kw = dict(min_size=4, max_size=32, shift=2, lam=200.0)
    plan = ctx.search_plan(128, 128, mb.make_params(**kw))
    try:
        gh, gl, gr, gc = plan.encode(img, allowed_modes=(1, 1, 1, 1))
    finally:
        plan.close()
    oh, ol, orr, osev, owev = orc.encode(img, orc.make_params(**kw), allowed_modes=(1, 1, 1, 1))
    assert bytes(gh) == bytes(oh)
    assert gl.tobytes() == ol.tobytes() and gr.tobytes() == orr.tobytes()
