"""The allocation-free level search (mars_search_blocks_noalloc), for callers that cannot
allocate device memory (real-time pipelines, plug-ins whose host owns all device memory,
fixed device-memory budgets).  Its scratch is a fixed 16 MiB array inside the library; its
results must equal the allocating entry point's, bit for bit, call after call, up to the
documented limit (a 512 x 512 plane at every block size), and the oracle's on the full
512 x 512 stride-2 level of the throughput workload.

Collected last on purpose (file name): a failure here leaves every other test run."""
import hashlib
import json
import os

import numpy as np
import pytest

import mars_b200 as mb
from mars_b200 import synthetic

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fullsize_512.json")


def _grid(w, h, size):
    import torch
    r, c = np.meshgrid(np.arange(h // size) * size, np.arange(w // size) * size, indexing="ij")
    return (torch.from_numpy(r.ravel().astype(np.int32)).cuda(),
            torch.from_numpy(c.ravel().astype(np.int32)).cuda())


def _run(fn_name, ctx, d_img, w, h, size, shift, p, rows, cols, stream=None):
    import torch
    out = torch.zeros((len(rows), 80), dtype=torch.uint8, device="cuda")
    torch.cuda.synchronize()
    if fn_name == "noalloc":
        rc = mb.lib().mars_search_blocks_noalloc(d_img.data_ptr(), w, h, size, shift, mb.C.byref(p),
                                                 rows.data_ptr(), cols.data_ptr(), len(rows),
                                                 out.data_ptr(), stream)
    else:
        rc = mb.lib().mars_search_blocks_device(ctx.handle, d_img.data_ptr(), w, h, size, shift,
                                                mb.C.byref(p), rows.data_ptr(), cols.data_ptr(),
                                                len(rows), out.data_ptr())
    mb.check(rc)
    torch.cuda.synchronize()
    return out.cpu().numpy().view(mb.CANDIDATE_DTYPE).ravel()


@pytest.fixture(scope="module")
def ctx():
    c = mb.Context(0)
    yield c
    c.close()


def test_noalloc_matches_allocating_entry_point_on_consecutive_calls(ctx):
    import torch
    cases = [(synthetic.gray(192, 160, 21), 4, 2), (synthetic.gray(256, 224, 22), 8, 4),
             (synthetic.gray(192, 160, 23), 4, 2)]
    for img, size, shift in cases:  # consecutive calls share (and reuse) the scratch
        h, w = img.shape
        d_img = torch.from_numpy(img).cuda()
        rows, cols = _grid(w, h, size)
        p = mb.make_params(shift=shift)
        a = _run("noalloc", None, d_img, w, h, size, shift, p, rows, cols)
        b = _run("device", ctx, d_img, w, h, size, shift, p, rows, cols)
        assert a.tobytes() == b.tobytes(), (size, shift)
        assert a["valid"].all()


@pytest.mark.parametrize("size", [2, 4, 8, 16, 32, 64])
def test_noalloc_full_512_plane_every_block_size(ctx, size):
    """The documented limit: every aligned block of a 512 x 512 plane at every block size,
    stride 2, fits the scratch and equals the allocating entry point."""
    import torch
    img = synthetic.gray(512, 512, 3)
    d_img = torch.from_numpy(img).cuda()
    rows, cols = _grid(512, 512, size)
    p = mb.make_params(min_size=min(size, 4), max_size=max(size, 4), shift=2)
    for _ in range(2):
        a = _run("noalloc", None, d_img, 512, 512, size, 2, p, rows, cols)
        b = _run("device", ctx, d_img, 512, 512, size, 2, p, rows, cols)
        assert a.tobytes() == b.tobytes(), size


def test_noalloc_equals_oracle_on_full_512_level():
    """Every 4 x 4 block of the 512 x 512 seed-1 plane at stride 2 against the oracle's
    digest of the same level (tests/golden/make_fullsize.py)."""
    import torch
    with open(GOLDEN) as f:
        want = json.load(f)["search"]["1"]["4"]
    img = synthetic.gray(512, 512, 1)
    d_img = torch.from_numpy(img).cuda()
    rows, cols = _grid(512, 512, 4)
    a = _run("noalloc", None, d_img, 512, 512, 4, 2, mb.make_params(shift=2), rows, cols)
    assert hashlib.sha256(a.tobytes()).hexdigest() == want["sha256"]


def test_noalloc_on_a_torch_stream_and_on_planes_without_domains(ctx):
    import torch
    img = synthetic.gray(256, 256, 4)
    d_img = torch.from_numpy(img).cuda()
    rows, cols = _grid(256, 256, 8)
    p = mb.make_params(shift=2)
    s = torch.cuda.Stream()
    a = _run("noalloc", None, d_img, 256, 256, 8, 2, p, rows, cols, s.cuda_stream)
    b = _run("device", ctx, d_img, 256, 256, 8, 2, p, rows, cols)
    assert a.tobytes() == b.tobytes()
    # A plane narrower than two blocks has no legal domain: every record comes back invalid
    # (the search's None), written without a kernel launch.
    small = torch.from_numpy(synthetic.gray(24, 40, 5)).cuda()
    rows, cols = _grid(24, 40, 16)
    out = _run("noalloc", None, small, 24, 40, 16, 2, mb.make_params(max_size=16, shift=2),
               rows, cols)
    assert not out["valid"].any()


def test_noalloc_rejects_searches_beyond_its_scratch():
    import torch
    img = np.zeros((2048, 2048), dtype=np.uint8)
    d_img = torch.from_numpy(img).cuda()
    rows = torch.zeros(64, dtype=torch.int32, device="cuda")
    cols = torch.arange(64, dtype=torch.int32, device="cuda") * 4
    out = torch.zeros((64, 80), dtype=torch.uint8, device="cuda")
    p = mb.make_params(shift=2)
    rc = mb.lib().mars_search_blocks_noalloc(d_img.data_ptr(), 2048, 2048, 4, 2, mb.C.byref(p),
                                             rows.data_ptr(), cols.data_ptr(), 64, out.data_ptr(),
                                             None)
    assert rc == -1
    assert b"scratch" in mb.lib().mars_last_error()
