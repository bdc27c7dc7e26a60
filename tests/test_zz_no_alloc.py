"""The allocation-free level search (mars_search_blocks_noalloc), for callers that cannot
allocate device memory (real-time pipelines, plug-ins whose host owns all device memory,
fixed device-memory budgets).  Its scratch is a fixed 16 MiB array inside the library; its
results must equal the allocating entry point's, bit for bit, call after call.

Collected last on purpose (file name): a failure here leaves every other test run."""
import numpy as np
import pytest

import mars_b200 as mb
from mars_b200 import synthetic

pytestmark = pytest.mark.gpu


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


def test_noalloc_matches_allocating_entry_point_on_consecutive_calls():
    import torch
    ctx = mb.Context(0)
    try:
        cases = [(synthetic.gray(192, 160, 21), 4, 2), (synthetic.gray(256, 224, 22), 8, 4),
                 (synthetic.gray(192, 160, 23), 4, 2)]
        for img, size, shift in cases:  # consecutive calls share (and reuse) the scratch
            h, w = img.shape
            d_img = torch.from_numpy(img).cuda()
            r, c = np.meshgrid(np.arange(h // size) * size, np.arange(w // size) * size,
                               indexing="ij")
            rows = torch.from_numpy(r.ravel().astype(np.int32)).cuda()
            cols = torch.from_numpy(c.ravel().astype(np.int32)).cuda()
            p = mb.make_params(shift=shift)
            a = _run("noalloc", None, d_img, w, h, size, shift, p, rows, cols)
            b = _run("device", ctx, d_img, w, h, size, shift, p, rows, cols)
            assert a.tobytes() == b.tobytes(), (size, shift)
            assert a["valid"].all()
    finally:
        ctx.close()


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
