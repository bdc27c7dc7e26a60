"""The library's host codec on the CPU: mars_b200/csrc/codec.cpp (walk, walk_rd, the rate
snapshot, price.hpp's best_mode_leaf run as one lane, the host thread pool) built with the
oracle's search as its provider (tests/codec_host_harness.cpp), against the oracle's own
encode_image_with_search, bit-exact: leaves, mode-3 levels and both eval counters.  Each
case runs twice: the walk pricing node by node, and every node priced up front through the
batch interface the device pricer uses (price_all / PricedNodes)."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import mars_b200 as mb
from mars_b200 import synthetic
from oracle import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    orc.lib()  # liboracle.so built
    out = str(tmp_path_factory.mktemp("codec_host") / "codec_host.so")
    csrc = os.path.join(ROOT, "mars_b200", "csrc")
    cmd = ["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
           "-pthread", "-o", out, os.path.join(ROOT, "tests", "codec_host_harness.cpp"),
           os.path.join(csrc, "codec.cpp"), os.path.join(csrc, "format.cpp"),
           "-L" + os.path.join(ROOT, "oracle"), "-loracle",
           "-Wl,-rpath," + os.path.join(ROOT, "oracle")]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr[-3000:]
    lib = C.CDLL(out)
    vp, sz = C.c_void_p, C.c_size_t
    lib.host_encode.argtypes = [vp, C.c_uint32, C.c_uint32, vp, vp, C.c_int, vp, vp, sz, vp, vp,
                                sz, vp, vp]
    lib.host_encode.restype = C.c_int
    return lib


def host_encode(lib, img, params, options, batch):
    a = np.ascontiguousarray(img, dtype=np.uint8)
    h, w = a.shape
    cap = w * h
    leaves = np.zeros(cap, dtype=mb.LEAF_DTYPE)
    res = np.zeros(cap, dtype=np.int32)
    hdr, cnt = mb.Header(), mb.Counters()
    nl, nr = C.c_size_t(), C.c_size_t()
    rc = lib.host_encode(a.ctypes.data, w, h, C.addressof(params), C.addressof(options),
                         int(batch), C.addressof(hdr), leaves.ctypes.data, cap, C.addressof(nl),
                         res.ctypes.data, cap, C.addressof(nr), C.addressof(cnt))
    assert rc == 0, rc
    return hdr, leaves[:nl.value], res[:nr.value], cnt


# (plane (w, h, seed), params, allowed_modes, options)
CASES = [
    ((96, 80, 101), dict(min_size=4, max_size=16, shift=2, lam=200.0), (1, 0, 1, 0), {}),
    ((96, 72, 102), dict(min_size=4, max_size=16, shift=2, lam=60.0), (1, 1, 1, 1),
     dict(residual_qstep=4.0)),
    ((80, 64, 103), dict(min_size=2, max_size=16, shift=2, lam=20.0), (1, 1, 1, 1), {}),
    ((88, 72, 104), dict(min_size=4, max_size=16, shift=4, lam=150.0), (0, 0, 0, 1), {}),
    ((96, 80, 105), dict(min_size=4, max_size=16, shift=2, lam=200.0), (1, 0, 1, 1),
     dict(rd_candidates=3)),
    ((96, 80, 106), dict(min_size=4, max_size=16, shift=2, lam=120.0), (1, 1, 1, 1),
     dict(adaptive_density=True)),
    ((72, 56, 107), dict(min_size=4, max_size=16, shift=2, lam=250.0), (1, 1, 1, 1),
     dict(residual_adaptive=True)),
    ((66, 40, 108), dict(min_size=1, max_size=16, shift=2, lam=200.0), (1, 1, 1, 0), {}),
    ((96, 80, 109), dict(min_size=4, max_size=16, shift=2), (1, 0, 1, 0), {}),
]


@pytest.mark.parametrize("batch", [False, True])
@pytest.mark.parametrize("case", range(len(CASES)))
def test_host_codec_matches_oracle(harness, case, batch):
    (w, h, seed), kw, modes, extra = CASES[case]
    img = synthetic.gray(w, h, seed)
    opts = mb.Options((C.c_uint8 * 4)(*modes), int(extra.get("adaptive_density", False)),
                      int(extra.get("residual_adaptive", False)),
                      float(extra.get("residual_qstep", 0.0)), 0,
                      int(extra.get("rd_candidates", 1)))
    gh, gl, gr, gc = host_encode(harness, img, mb.make_params(**kw), opts, batch)
    oh, ol, orr, osev, owev = orc.encode(img, orc.make_params(**kw), allowed_modes=modes, **extra)
    assert bytes(gh) == bytes(oh)
    assert gl.tobytes() == ol.tobytes()
    assert gr.tobytes() == orr.tobytes()
    assert (gc.search_evals, gc.warmup_evals) == (osev, owev)


@pytest.mark.parametrize("threads", ["1", "3", "32"])
def test_host_pool_sizes_give_the_same_encode(harness, monkeypatch, threads):
    img = synthetic.gray(112, 96, 110)
    kw = dict(min_size=4, max_size=16, shift=2, lam=200.0)
    opts = mb.Options((C.c_uint8 * 4)(1, 1, 1, 1), 0, 0, 0.0, 0, 1)
    monkeypatch.setenv("MARS_HOST_THREADS", threads)
    gh, gl, gr, gc = host_encode(harness, img, mb.make_params(**kw), opts, False)
    oh, ol, orr, osev, owev = orc.encode(img, orc.make_params(**kw), allowed_modes=(1, 1, 1, 1))
    assert gl.tobytes() == ol.tobytes() and gr.tobytes() == orr.tobytes()
