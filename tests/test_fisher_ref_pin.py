"""The Fisher classification pinned to the reference's own C code.

oracle/_ref/libmars1_fisher.so is the reference's 1998 classifier (reference/mars1:
FisherIndexing, newclass, variance_class, flips) compiled from its sources by
`make -C oracle ref`.  On square planes (where that code's contraction() is the intended
one), every domain position's bucket (class * 24 + variance class) and canonicalising
isometry from the oracle's restatement of crates/mars-search/src/classify.rs must equal the
C code's, and every range block's search must read the bucket the C code assigns to the
range: its eval count is that bucket's length (the first non-empty bucket when it is empty)
and its winner is a domain of that bucket with isometry MAPPING[range iso][domain iso]
(crates/mars-search/src/fisher.rs:30-78; coding_func.c FisherCoding).

Skipped when the reference build is absent (it is built in a container that has the
reference checkout and travels with the tree)."""
import ctypes as C
import os

import numpy as np
import pytest

from mars_b200 import synthetic
from oracle import oracle as orc
from tests.golden_data import fixture_images

LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                   "libmars1_fisher.so")

# crates/mars-search/src/tables.rs MAPPING (Mars 1 globals.h): candidate isometry for a
# (range isometry, domain isometry) pair.
MAPPING = np.array([[0, 1, 2, 3, 4, 5, 6, 7], [2, 0, 3, 1, 7, 6, 4, 5], [1, 3, 0, 2, 6, 7, 5, 4],
                    [3, 2, 1, 0, 5, 4, 7, 6], [4, 7, 6, 5, 0, 3, 2, 1], [5, 6, 7, 4, 3, 0, 1, 2],
                    [6, 4, 5, 7, 1, 2, 0, 3], [7, 5, 4, 6, 2, 1, 3, 0]])


def ref_lib():
    if not os.path.exists(LIB):
        pytest.skip("oracle/_ref/libmars1_fisher.so not built (no reference checkout)")
    lib = C.CDLL(LIB)
    lib.m1_fisher_domains.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.POINTER(C.c_int)]
    lib.m1_fisher_range.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                    C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
    return lib


def c_domains(img, size, shift):
    """(bucket, iso, counts, first non-empty bucket) of every domain position, from C."""
    lib = ref_lib()
    a = np.ascontiguousarray(img, dtype=np.uint8)
    h, w = a.shape
    n = ((h - 2 * size) // shift + 1) * ((w - 2 * size) // shift + 1)
    bucket = np.zeros(n, np.uint8)
    iso = np.zeros(n, np.uint8)
    counts = np.zeros(72, np.uint32)
    first = C.c_int()
    rc = lib.m1_fisher_domains(a.ctypes.data, w, h, size, shift, bucket.ctypes.data,
                               iso.ctypes.data, counts.ctypes.data, C.byref(first))
    assert rc == 0
    return bucket, iso, counts, first.value


def c_ranges(img, size, rows, cols):
    """(bucket key, isometry) of each range block, from C's FisherCoding classification."""
    lib = ref_lib()
    a = np.ascontiguousarray(img, dtype=np.uint8)
    keys, isos = [], []
    cl, va, im = C.c_int(), C.c_int(), C.c_int()
    for r, c in zip(rows, cols):
        assert lib.m1_fisher_range(a.ctypes.data, a.shape[1], size, int(r), int(c), C.byref(cl),
                                   C.byref(va), C.byref(im)) == 0
        keys.append(cl.value * 24 + va.value)
        isos.append(im.value)
    return np.array(keys), np.array(isos)


def grid(w, h, size):
    r, c = np.meshgrid(np.arange(0, h - size + 1, size), np.arange(0, w - size + 1, size),
                       indexing="ij")
    return r.ravel().astype(np.uint32), c.ravel().astype(np.uint32)


def expected_reads(img, size, shift):
    """Per range block of the aligned grid: the bucket it reads, per the C classifier, its
    length, and the range's isometry; with the C domain classification."""
    h, w = img.shape
    bucket, diso, counts, first = c_domains(img, size, shift)
    rows, cols = grid(w, h, size)
    keys, risos = c_ranges(img, size, rows, cols)
    eff = np.where(counts[keys] > 0, keys, first)
    return rows, cols, eff, counts[eff], risos, bucket, diso


def square_planes():
    imgs, _ = fixture_images()
    out = [(name, im) for name, im in imgs.items() if im.shape[0] == im.shape[1]]
    out += [(f"synthetic{s}", synthetic.gray(256, 256, s)) for s in (1, 2)]
    return out


PLANES = square_planes()


@pytest.mark.parametrize("name,img", PLANES, ids=[p[0] for p in PLANES])
@pytest.mark.parametrize("size,shift", [(4, 2), (8, 4), (16, 2)])
def test_domain_classes_equal_the_reference_c_code(name, img, size, shift):
    bucket, iso, _, _ = c_domains(img, size, shift)
    ob, oi = orc.fisher_classify_domains(img, size, shift)
    assert np.array_equal(ob, bucket), f"{name}: buckets differ at {np.nonzero(ob != bucket)[0][:5]}"
    assert np.array_equal(oi, iso), f"{name}: isometries differ at {np.nonzero(oi != iso)[0][:5]}"


# The range-side check runs the oracle's classified search; the 256 x 256 planes keep it to
# seconds (the 512 x 512 binary sierpinski plane puts most domains in a few buckets).
RANGE_PLANES = [p for p in PLANES if p[1].shape[0] <= 256]


@pytest.mark.parametrize("name,img", RANGE_PLANES, ids=[p[0] for p in RANGE_PLANES])
@pytest.mark.parametrize("size,shift", [(4, 2), (8, 2)])
def test_range_reads_the_bucket_the_reference_c_code_assigns(name, img, size, shift):
    h, w = img.shape
    rows, cols, eff, length, risos, bucket, diso = expected_reads(img, size, shift)
    out, ev = orc.fisher_search_blocks(img, size, shift, orc.make_params(shift=shift), rows, cols)
    assert np.array_equal(ev, length), f"{name}: eval counts differ from the C bucket lengths"
    ncol = (w - 2 * size) // shift + 1
    pos = (out["dom_row"] // shift) * ncol + out["dom_col"] // shift
    assert out["valid"].all()
    assert np.array_equal(bucket[pos], eff), f"{name}: a winner lies outside its C bucket"
    assert np.array_equal(out["isometry"], MAPPING[risos, diso[pos]])


def _iso_permute(block, k):
    """permute_range (crates/mars-codec/src/encode.rs:833-842) with isometry::map
    (crates/mars-codec/src/isometry.rs:7-19): out[u, v] = block[map_k(u, v)]."""
    s = block.shape[0]
    u, v = np.meshgrid(np.arange(s), np.arange(s), indexing="ij")
    i, j = [(u, v), (s - 1 - v, u), (v, s - 1 - u), (s - 1 - u, s - 1 - v), (u, s - 1 - v),
            (s - 1 - u, v), (v, u), (s - 1 - v, s - 1 - u)][k]
    return block[i, j]


def _flips(block, iso):
    """flips (crates/mars-search/src/classify.rs; Mars 1 coding_func.c:1200-1247):
    out[i, j] = block[source of (i, j) under iso]."""
    s = block.shape[0]
    i, j = np.meshgrid(np.arange(s), np.arange(s), indexing="ij")
    si, sj = [(i, j), (j, s - i - 1), (s - j - 1, i), (s - i - 1, s - j - 1), (i, s - j - 1),
              (s - i - 1, j), (j, i), (s - j - 1, s - i - 1)][iso]
    return block[si, sj]


@pytest.mark.parametrize("size", [2, 4, 8, 16])
def test_canonical_orientation_turns_every_bucket_into_one_product(size):
    """For every (range isometry, domain isometry) pair the classified search's cross term
    sum R[MAPPING[ri][di](u, v)] * D[u, v] equals sum flips(R, ri) * flips(D, di): with both
    operands brought to their canonical orientation, the pairs of one bucket are one plain
    matrix product (no per-pair isometry)."""
    rng = np.random.default_rng(size)
    for ri in range(8):
        for di in range(8):
            r = rng.integers(0, 256, (size, size))
            d = rng.integers(0, 1021, (size, size))
            want = int((_iso_permute(r, MAPPING[ri, di]) * d).sum())
            assert int((_flips(r, ri) * _flips(d, di)).sum()) == want, (ri, di)
