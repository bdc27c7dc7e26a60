"""Oracle records for a sample of the 4096x4096 search (the uneven batch's large plane).

A whole 4096x4096 exhaustive search is 4.65e13 evals: hours for the CPU oracle.  This
script takes a seeded sample of RD-quadtree nodes of the synthetic plane
(mars_b200.synthetic.gray(4096, 4096, 99); block sizes 32, 16, 8, 4; domain stride 2).  The
sample includes the last block row and column and the plane's corners.  For each node it
runs the CPU oracle (oracle/, the reference's search_top_k + fit_f64 restated,
crates/mars-codec/src/encode.rs:695-788) over every domain of the plane.  It writes the
candidate records (80-byte mars_candidate, hex) and the eval counts to sample_4096.json.
tests/test_gpu_fullsize.py compares the device search of the same nodes with them, on both
correlation paths.  About 2 minutes on 8 host cores.

  python tests/golden/make_sample_4096.py
"""
from __future__ import annotations

import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

SIDE = 4096
SEED = 99
SHIFT = 2
SAMPLE = {32: 8, 16: 12, 8: 16, 4: 24}  # nodes per block size


def sample_nodes(size: int, count: int, rng) -> list[tuple[int, int]]:
    """`count` distinct aligned block origins: the four corners, then random ones."""
    last = SIDE - size
    nodes = [(0, 0), (0, last), (last, 0), (last, last)]
    while len(nodes) < count:
        rc = (int(rng.integers(0, SIDE // size)) * size, int(rng.integers(0, SIDE // size)) * size)
        if rc not in nodes:
            nodes.append(rc)
    return nodes


def main() -> int:
    import numpy as np
    from mars_b200 import synthetic
    from oracle import oracle as orc

    img = synthetic.gray(SIDE, SIDE, SEED)
    params = orc.make_params(min_size=4, max_size=32, shift=SHIFT)
    rng = np.random.default_rng(4096)
    out = {"generator": "tests/golden/make_sample_4096.py", "side": SIDE, "seed": SEED,
           "shift": SHIFT, "record": "mars_candidate, 80 bytes, hex", "levels": {}}
    for size, count in SAMPLE.items():
        nodes = sample_nodes(size, count, rng)
        rows = np.array([r for r, _ in nodes], np.uint32)
        cols = np.array([c for _, c in nodes], np.uint32)
        t0 = time.time()
        cands, evals = orc.search_blocks(img, size, SHIFT, params, rows, cols)
        out["levels"][str(size)] = {"rows": rows.tolist(), "cols": cols.tolist(),
                                    "records": [c.tobytes().hex() for c in cands],
                                    "evals": [int(e) for e in evals]}
        print(f"size {size}: {count} nodes, {time.time() - t0:.1f} s", flush=True)
    with open(os.path.join(HERE, "sample_4096.json"), "w") as f:
        json.dump(out, f, indent=1)
        f.write("\n")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
