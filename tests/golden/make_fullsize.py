"""Digests of the oracle's search and encode on the full 512x512 exhaustive workload.

The throughput workload searches every RD-quadtree node of a 512x512 synthetic plane
(mars_b200.synthetic.gray, seeds 1-8; block sizes 32, 16, 8, 4; domain stride 2).  This
script runs the CPU oracle (oracle/, the reference's search_top_k + fit_f64 restated,
crates/mars-codec/src/encode.rs:695-788) on every one of those nodes and writes, per seed
and block size, the SHA-256 of the oracle's candidate records (80-byte mars_candidate
records, aligned blocks in row-major order) and the eval total.  For seed 1 it also writes
the SHA-256 and length of the `.mars` v0 stream of the oracle's RD encode at lambda 50, 200
and 800 (modes {0, 2}, sizes 32..4, stride 2), serialised by the library's host writer,
which the reference's own stream hashes pin (tests/test_mars_format.py).

The output, fullsize_512.json, is committed; tests/test_gpu_fullsize.py compares the GPU
search plan and the GPU encode with it.  About 20 minutes on 8 host cores.

  python tests/golden/make_fullsize.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

SIDE = 512
SIZES = (32, 16, 8, 4)
SHIFT = 2
SEEDS = tuple(range(1, 9))
LAMBDAS = (50.0, 200.0, 800.0)
MODES = (1, 0, 1, 0)


def main() -> int:
    import mars_b200 as mb
    from mars_b200 import synthetic
    from oracle import oracle as orc

    params = orc.make_params(min_size=4, max_size=32, shift=SHIFT)
    out = {"generator": "tests/golden/make_fullsize.py", "side": SIDE, "sizes": list(SIZES),
           "shift": SHIFT, "record": "mars_candidate, 80 bytes, aligned blocks row-major",
           "search": {}, "encode": {}}
    for seed in SEEDS:
        img = synthetic.gray(SIDE, SIDE, seed)
        per = {}
        for size in SIZES:
            t0 = time.time()
            cands, evals = orc.search_grid(img, size, SHIFT, params)
            per[str(size)] = {"sha256": hashlib.sha256(cands.tobytes()).hexdigest(),
                              "evals": int(evals.sum()), "blocks": int(len(cands))}
            print(f"seed {seed} size {size}: {time.time() - t0:.1f} s", flush=True)
        out["search"][str(seed)] = per

    img = synthetic.gray(SIDE, SIDE, 1)
    for lam in LAMBDAS:
        t0 = time.time()
        p = orc.make_params(min_size=4, max_size=32, shift=SHIFT, lam=lam)
        hdr, leaves, res, sev, wev = orc.encode(img, p, allowed_modes=MODES)
        mhdr = mb.Header(*[getattr(hdr, f) for f, _ in mb.Header._fields_])
        data = mb.format_write(mhdr, leaves, res)
        out["encode"][str(int(lam))] = {"seed": 1, "modes": list(MODES), "bytes": len(data),
                                        "sha256": hashlib.sha256(data).hexdigest(),
                                        "leaves": int(len(leaves)), "search_evals": int(sev),
                                        "warmup_evals": int(wev)}
        print(f"encode lambda {lam}: {time.time() - t0:.1f} s", flush=True)

    with open(os.path.join(HERE, "fullsize_512.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote fullsize_512.json")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
