"""Loaders for the committed golden fixtures (generated by tests/golden/make_golden.py)."""
import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def mars1_manifest():
    with open(os.path.join(GOLDEN, "mars1_manifest.json")) as f:
        return json.load(f)


def mars1_bytes(entry) -> bytes:
    with open(os.path.join(GOLDEN, "mars1", entry["file"]), "rb") as f:
        return f.read()


def fixture_images():
    with open(os.path.join(GOLDEN, "images.json")) as f:
        meta = json.load(f)["images"]
    arrs = np.load(os.path.join(GOLDEN, "images.npz"))
    return {m["name"]: arrs[m["name"]] for m in meta}, meta


def provider_pattern_16():
    """The 16x16 image of crates/mars-codec/tests/search_provider.rs:13-27."""
    i = np.arange(256)
    v = np.where(i % 16 < 8, 100, (i * 37 + i // 16 * 13) % 256)
    return v.astype(np.uint8).reshape(16, 16)
