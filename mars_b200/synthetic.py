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
