"""Seeded synthetic test planes for the Mars search benchmarks.

The benchmark workloads are quoted on seeded synthetic 8-bit images: the sum of 6 random
2-D sinusoids (periods 8-128 px, amplitudes 20-40), 12 random axis-aligned rectangles of
uniform value 0-255, and Gaussian noise of sigma 6, clipped to 0-255.  Two choices are left
open by that description and are fixed here once (version 1 of this generator):

  * the sinusoids sit on a base level of 128;
  * rectangles overwrite the sinusoid field (they are not added to it), each with a side
    drawn uniformly from [8, max(8, dim // 4)], and the noise is added afterwards;
  * the generator is numpy's PCG64 seeded with the image seed; pixels are rounded to the
    nearest integer before clipping.

`PINNED_SHA256` pins the outputs so any change to this file shows up as a test failure.
"""
from __future__ import annotations

import hashlib

import numpy as np

GENERATOR_VERSION = 1


def gray(width: int, height: int, seed: int) -> np.ndarray:
    """One synthetic 8-bit grayscale plane, shape (height, width)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    yy, xx = np.mgrid[0:height, 0:width].astype(np.float64)
    field = np.full((height, width), 128.0)
    for _ in range(6):
        period = rng.uniform(8.0, 128.0)
        theta = rng.uniform(0.0, np.pi)
        phase = rng.uniform(0.0, 2.0 * np.pi)
        amp = rng.uniform(20.0, 40.0)
        k = 2.0 * np.pi / period
        field += amp * np.sin(k * (xx * np.cos(theta) + yy * np.sin(theta)) + phase)
    for _ in range(12):
        rh = int(rng.integers(8, max(9, height // 4 + 1)))
        rw = int(rng.integers(8, max(9, width // 4 + 1)))
        r0 = int(rng.integers(0, max(1, height - rh + 1)))
        c0 = int(rng.integers(0, max(1, width - rw + 1)))
        field[r0:r0 + rh, c0:c0 + rw] = rng.uniform(0.0, 255.0)
    field += rng.normal(0.0, 6.0, size=(height, width))
    return np.clip(np.rint(field), 0, 255).astype(np.uint8)


def rgb(width: int, height: int, seed: int) -> np.ndarray:
    """Synthetic RGB: the gray generator per channel, then a random 3x3 channel mix.
    Shape (height, width, 3), uint8."""
    chans = np.stack([gray(width, height, seed * 3 + c + 1000) for c in range(3)], axis=-1)
    rng = np.random.Generator(np.random.PCG64(seed + 7777))
    mix = rng.uniform(0.0, 1.0, size=(3, 3))
    mix /= mix.sum(axis=1, keepdims=True)
    out = chans.astype(np.float64) @ mix.T
    return np.clip(np.rint(out), 0, 255).astype(np.uint8)


def sha256(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def batch_sides(count: int, seed: int) -> list[int]:
    """Side lengths of the uneven batch: uniform over {128, 256, 384, 512, 768, 1024}."""
    rng = np.random.Generator(np.random.PCG64(seed))
    choices = np.array([128, 256, 384, 512, 768, 1024])
    return [int(x) for x in rng.choice(choices, size=count)]


def quadtree_leaves(width: int, height: int, seed: int, max_size: int = 32, min_size: int = 4,
                    split_p: float = 0.6, shift: int = 2, bits_alfa: int = 4, bits_beta: int = 7,
                    p_flat: float = 0.15, p_affine: float = 0.1) -> np.ndarray:
    """A synthetic decode map: a random quadtree partition of the plane into leaves of
    sizes max_size..min_size (each node split with probability split_p), in depth-first
    order within each top block as the encoder emits them.  Leaves are mode 0 (flat) with
    probability p_flat, mode 1 (affine) with p_affine, otherwise mode 2 with a random
    domain on the stride grid, a random isometry and qalfa in 1..2^bits_alfa.  Returns a
    structured array of the library's leaf dtype (fields row, col, size, mode, qalfa, qbeta,
    isometry, dom_row, dom_col, qgx, qgy)."""
    dtype = np.dtype([(n, "<u4") for n in (
        "row", "col", "size", "mode", "qalfa", "qbeta", "isometry", "dom_row", "dom_col")] + [
        ("qgx", "<i4"), ("qgy", "<i4")])
    rng = np.random.Generator(np.random.PCG64(seed))
    tr, tc = np.mgrid[0:height - max_size + 1:max_size, 0:width - max_size + 1:max_size]
    r, c = tr.ravel().astype(np.int64), tc.ravel().astype(np.int64)
    parts = []
    size = max_size
    while len(r):
        split = (rng.random(len(r)) < split_p) if size > min_size else np.zeros(len(r), bool)
        parts.append((r[~split], c[~split], np.full((~split).sum(), size, np.int64)))
        r, c = r[split], c[split]
        half = size // 2
        r = np.concatenate([r, r, r + half, r + half])
        c = np.concatenate([c, c + half, c, c + half])
        size = half
    rows = np.concatenate([p[0] for p in parts])
    cols = np.concatenate([p[1] for p in parts])
    sizes = np.concatenate([p[2] for p in parts])
    # Depth-first order: top block, then the Morton code of the leaf within it.
    lr, lc = rows % max_size, cols % max_size
    morton = np.zeros(len(rows), np.int64)
    for b in range(int(max_size).bit_length()):
        morton |= ((lr >> b) & 1) << (2 * b + 1) | ((lc >> b) & 1) << (2 * b)
    tiles_across = (width + max_size - 1) // max_size
    key = ((rows // max_size) * tiles_across + cols // max_size) << 24 | morton
    order = np.argsort(key, kind="stable")
    rows, cols, sizes = rows[order], cols[order], sizes[order]
    n = len(rows)
    out = np.zeros(n, dtype)
    out["row"], out["col"], out["size"] = rows, cols, sizes
    kind = rng.random(n)
    mode = np.where(kind < p_flat, 0, np.where(kind < p_flat + p_affine, 1, 2))
    out["mode"] = mode
    out["qbeta"] = rng.integers(0, (1 << bits_beta), n)
    dom_rows = (height - 2 * sizes) // shift + 1
    dom_cols = (width - 2 * sizes) // shift + 1
    ok = (dom_rows > 0) & (dom_cols > 0)
    fractal = (mode == 2) & ok
    out["mode"][(mode == 2) & ~ok] = 0
    out["qalfa"] = np.where(fractal, rng.integers(1, (1 << bits_alfa) + 1, n), 0)
    out["isometry"] = np.where(fractal, rng.integers(0, 8, n), 0)
    pick_r = np.floor(rng.random(n) * np.maximum(dom_rows, 1)).astype(np.int64)
    pick_c = np.floor(rng.random(n) * np.maximum(dom_cols, 1)).astype(np.int64)
    out["dom_row"] = np.where(fractal, pick_r * shift, 0)
    out["dom_col"] = np.where(fractal, pick_c * shift, 0)
    affine = mode == 1
    out["qgx"] = np.where(affine, rng.integers(-96, 97, n), 0)
    out["qgy"] = np.where(affine, rng.integers(-96, 97, n), 0)
    return out
