"""Properties of the oracle's Fisher restatement (crates/mars-search/src/fisher.rs,
classify.rs) that hold whatever the image: a block's eval count is the length of the bucket
it reads, its winner comes from that bucket, and a plane whose domains all classify alike
sends every block to that one bucket (the empty-bucket fallback, fisher.rs:42-54)."""
import numpy as np

from mars_b200 import synthetic
from oracle import oracle as orc
from tests.golden_data import fixture_images


def _grid(w, h, size):
    r, c = np.meshgrid(np.arange(0, h - size + 1, size), np.arange(0, w - size + 1, size),
                       indexing="ij")
    return r.ravel().astype(np.uint32), c.ravel().astype(np.uint32)


def test_evals_are_the_winners_bucket_length():
    img = synthetic.gray(96, 80, 2)
    h, w = img.shape
    for size, shift in ((4, 2), (8, 2), (8, 4), (16, 2)):
        bucket, _ = orc.fisher_classify_domains(img, size, shift)
        counts = np.bincount(bucket, minlength=72)
        ncol = (w - 2 * size) // shift + 1
        rows, cols = _grid(w, h, size)
        out, ev = orc.fisher_search_blocks(img, size, shift, orc.make_params(shift=shift), rows,
                                           cols)
        assert out["valid"].all()
        pos = (out["dom_row"] // shift) * ncol + out["dom_col"] // shift
        assert np.array_equal(ev, counts[bucket[pos]])
        assert ev.sum() < len(rows) * len(bucket) * 8 / 20  # far fewer than exhaustive


def test_flat_plane_reads_one_bucket():
    imgs, _ = fixture_images()
    img = imgs["flat128"]
    h, w = img.shape
    bucket, iso = orc.fisher_classify_domains(img, 4, 2)
    assert len(set(bucket.tolist())) == 1 and (iso == 0).all()
    rows, cols = _grid(w, h, 4)
    _, ev = orc.fisher_search_blocks(img, 4, 2, orc.make_params(shift=2), rows, cols)
    assert (ev == len(bucket)).all()


def test_encode_counts_only_final_walk_searches():
    img = synthetic.gray(64, 64, 5)
    p = orc.make_params(min_size=4, max_size=16, shift=2, lam=100.0)
    _, _, _, sev_f, wev_f = orc.encode(img, p, allowed_modes=(1, 1, 1, 1), method="fisher")
    _, _, _, sev_e, wev_e = orc.encode(img, p, allowed_modes=(1, 1, 1, 1))
    assert wev_f == wev_e  # the rate warm-up stays exhaustive
    assert sev_f < sev_e
