"""Parity at the size the throughput is measured on: every RD-quadtree node of the 512x512
synthetic planes (seeds 1-8, block sizes 32..4, domain stride 2) through the graph-captured
search plan, against the oracle's digests of the same nodes (tests/golden/make_fullsize.py),
and the `.mars` bytes of seed 1's RD encodes at lambda 50 / 200 / 800.

At this size the tensor-core kernel meets what the small cases do not: many domain tiles per
CTA, M-splits merged by the finish kernel, survivor-queue drains across tiles.  The bar is
bit-exact: every 80-byte candidate record (f64 rms bit pattern and moments included) and
every eval count.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import mars_b200 as mb
from mars_b200 import synthetic

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "fullsize_512.json")


@pytest.fixture(scope="module")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def ctx():
    c = mb.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def plan(ctx, golden):
    p = ctx.search_plan(golden["side"], golden["side"],
                        mb.make_params(min_size=4, max_size=32, shift=golden["shift"]))
    yield p
    p.close()


def _level(table, side, size, shift):
    rows, cols = np.meshgrid(np.arange(side // size) * size, np.arange(side // size) * size,
                             indexing="ij")
    return table.search_many(rows.ravel(), cols.ravel(), size, shift)


def _check_table(table, golden, seed):
    side, shift = golden["side"], golden["shift"]
    want = golden["search"][str(seed)]
    for size in golden["sizes"]:
        cands, evals = _level(table, side, size, shift)
        w = want[str(size)]
        assert len(cands) == w["blocks"]
        assert int(evals.sum()) == w["evals"], (seed, size)
        got = hashlib.sha256(cands.tobytes()).hexdigest()
        assert got == w["sha256"], f"seed {seed} size {size}: node table differs from the oracle"


@pytest.mark.parametrize("seed", range(1, 9))
def test_plan_run_matches_oracle_digests(plan, golden, seed):
    img = synthetic.gray(golden["side"], golden["side"], seed)
    table = plan.run(img)
    try:
        _check_table(table, golden, seed)
    finally:
        table.close()


@pytest.mark.parametrize("seed", range(1, 9))
def test_plan_run_device_matches_oracle_digests(plan, golden, seed):
    import torch
    img = synthetic.gray(golden["side"], golden["side"], seed)
    d = torch.from_numpy(img).to("cuda:0")
    torch.cuda.synchronize()
    plan.run_device(d.data_ptr())
    table = plan.table()
    try:
        _check_table(table, golden, seed)
    finally:
        table.close()


@pytest.mark.parametrize("lam", [50, 200, 800])
def test_rd_encode_bytes_match_oracle(ctx, plan, golden, lam):
    want = golden["encode"][str(lam)]
    img = synthetic.gray(golden["side"], golden["side"], want["seed"])
    params = mb.make_params(min_size=4, max_size=32, shift=golden["shift"], lam=float(lam))
    modes = tuple(want["modes"])
    # One-shot encode (provider factory + host walks).
    hdr, leaves, res, cnt = ctx.encode(img, params, allowed_modes=modes)
    data = mb.format_write(hdr, leaves, res)
    assert (len(data), hashlib.sha256(data).hexdigest()) == (want["bytes"], want["sha256"])
    assert (cnt.search_evals, cnt.warmup_evals) == (want["search_evals"], want["warmup_evals"])
    # Planned encode: the search graph, then the warm-up walk, pricing and RD decisions on
    # the device.
    lp = ctx.search_plan(golden["side"], golden["side"], params)
    try:
        hdr2, leaves2, res2, cnt2 = lp.encode(img, allowed_modes=modes)
    finally:
        lp.close()
    data2 = mb.format_write(hdr2, leaves2, res2)
    assert hashlib.sha256(data2).hexdigest() == want["sha256"]
    assert (cnt2.search_evals, cnt2.warmup_evals) == (want["search_evals"], want["warmup_evals"])


# ---- the 4096x4096 plane of the uneven batch: a seeded sample of nodes (corners and border
# blocks included) searched over every domain of the plane, against the oracle's records
# (tests/golden/make_sample_4096.py).  At this size one block sweeps 4.1 M domain positions:
# thousands of domain tiles per CTA, 32-bit domain indices near 2^25, and, at 32 and 16, the
# split-digit operand over a 2048x2048 contracted plane.

SAMPLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sample_4096.json")


@pytest.fixture(scope="module")
def sample():
    with open(SAMPLE) as f:
        s = json.load(f)
    import torch
    s["plane"] = torch.from_numpy(synthetic.gray(s["side"], s["side"], s["seed"])).cuda()
    return s


@pytest.mark.parametrize("path", ["auto", "simt"])
@pytest.mark.parametrize("size", [32, 16, 8, 4])
def test_4096_sample_matches_oracle_records(ctx, sample, size, path):
    import torch
    side, shift = sample["side"], sample["shift"]
    lv = sample["levels"][str(size)]
    n = len(lv["rows"])
    ndom = ((side - 2 * size) // shift + 1) ** 2
    assert lv["evals"] == [8 * ndom] * n  # the exhaustive count, positions x 8
    rows = torch.tensor(lv["rows"], dtype=torch.int32, device="cuda")
    cols = torch.tensor(lv["cols"], dtype=torch.int32, device="cuda")
    out = torch.zeros((n, mb.CANDIDATE_DTYPE.itemsize), dtype=torch.uint8, device="cuda")
    p = mb.make_params(min_size=4, max_size=32, shift=shift)
    ctx.set_search_path(path)
    try:
        torch.cuda.synchronize()
        mb.check(mb.lib().mars_search_blocks_device(ctx.handle, sample["plane"].data_ptr(), side,
                                                    side, size, shift, mb.C.byref(p),
                                                    rows.data_ptr(), cols.data_ptr(), n,
                                                    out.data_ptr()))
        torch.cuda.synchronize()
    finally:
        ctx.set_search_path("auto")
    got = out.cpu().numpy()
    for i in range(n):
        assert got[i].tobytes().hex() == lv["records"][i], (size, lv["rows"][i], lv["cols"][i])
