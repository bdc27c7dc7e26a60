"""Pins the seeded synthetic generator (mars_b200/synthetic.py, version 1): any change to
it changes every benchmark input and shows up here."""
import numpy as np

from mars_b200 import synthetic

PINNED = {
    (256, 256, 0): "003a44a7f09a5c5d02a6d8d2197f0513d1bd640603993e00da5ee6209006e3d7",
    (512, 512, 1): "b524dbacf2898199eec742fc6dc162547b8549575163ad370291ec2c1186b4f3",
    (512, 512, 8): "f585feea50824af797e4534fb55a4553093ee742226ac8832f6ef00eb2201050",
    (96, 80, 0): "192964eb76007953cf7cb01e87f3d7b3fa23c2af82fc06460e3b2daa55679b35",
}


def test_generator_version():
    assert synthetic.GENERATOR_VERSION == 1


def test_pinned_gray_planes():
    for (w, h, seed), digest in PINNED.items():
        img = synthetic.gray(w, h, seed)
        assert img.shape == (h, w) and img.dtype == np.uint8
        assert synthetic.sha256(img) == digest


def test_rgb_and_batch_sides():
    assert synthetic.sha256(synthetic.rgb(768, 512, 1)) == \
        "776684e8c88d74540cf9bbc9460ce6a5499e946f6cb021ca7c6471e80e48c04b"
    assert synthetic.batch_sides(8, 5) == [768, 768, 128, 768, 384, 512, 512, 256]


def test_value_statistics():
    # The generator's intent: full-range content with flat rectangles and noise.
    img = synthetic.gray(512, 512, 1).astype(np.int64)
    assert img.min() == 0 or img.max() == 255
    assert 40 < img.std() < 100


def test_quadtree_leaves_pinned_and_valid():
    leaves = synthetic.quadtree_leaves(512, 512, 3)
    assert synthetic.sha256(leaves) == (
        "20e9e7684f2a54ad953c4c9137a03e3d256b8166345b32156f5dd632a58f1e4d")
    cover = np.zeros((512, 512), np.int32)
    for r, c, s in zip(leaves["row"], leaves["col"], leaves["size"]):
        cover[r:r + s, c:c + s] += 1
    assert (cover == 1).all()  # a partition of the plane
    frac = leaves["qalfa"] > 0
    assert (leaves["mode"][frac] == 2).all()
    assert (leaves["dom_row"][frac] + 2 * leaves["size"][frac] <= 512).all()
    assert (leaves["dom_col"][frac] + 2 * leaves["size"][frac] <= 512).all()
    assert (leaves["dom_row"] % 2 == 0).all() and (leaves["dom_col"] % 2 == 0).all()
    assert set(np.unique(leaves["mode"])) == {0, 1, 2}
