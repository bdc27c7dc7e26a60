"""Regenerates the committed golden fixtures from the reference checkout.

Run once in a container that has the reference checkout, named by --reference or the
MARS_REFERENCE environment variable; the outputs are committed, so the tests never read the
reference at run time.

  * mars1/<stem>.ifs + mars1_manifest.json -- the reference's 142 Mars 1 golden .ifs
    streams (fixtures/mars1/) with the pinned transform counts, stream SHA-256 and
    10-iteration decode SHA-256 from fixtures/mars1/manifest.toml.
  * images.npz + images.json -- the reference's 12 synthetic fixture images, regenerated
    by its own scripts/gen-fixtures.py (stdlib only, deterministic MT19937) and checked
    against the SHA-256s pinned in fixtures/images/manifest.toml.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile
import tomllib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("MARS_REFERENCE"))
    args = ap.parse_args()
    ref = args.reference
    if not ref:
        ap.error("name the reference checkout with --reference or MARS_REFERENCE")

    # --- Mars 1 .ifs streams and their pinned decode hashes
    with open(os.path.join(ref, "fixtures/mars1/manifest.toml"), "rb") as f:
        man = tomllib.load(f)
    out_dir = os.path.join(HERE, "mars1")
    os.makedirs(out_dir, exist_ok=True)
    keep = ("stem", "file", "image", "width", "height", "method", "t_rms", "min_size",
            "max_size", "shift", "bits_alfa", "bits_beta", "max_alfa", "ifs_bytes", "ifs_sha256",
            "transforms", "zero_alfa_transforms", "decode_iterative_sha256")
    entries = []
    for fx in man["fixture"]:
        src = os.path.join(ref, "fixtures/mars1", fx["file"])
        shutil.copyfile(src, os.path.join(out_dir, fx["file"]))
        entries.append({k: fx[k] for k in keep if k in fx})
    with open(os.path.join(HERE, "mars1_manifest.json"), "w") as f:
        json.dump({"source": "fixtures/mars1/manifest.toml", "decode_iterations": 10,
                   "fixtures": entries}, f, indent=1)

    # --- synthetic fixture images, regenerated by the reference's own generator
    with open(os.path.join(ref, "fixtures/images/manifest.toml"), "rb") as f:
        imman = tomllib.load(f)
    with tempfile.TemporaryDirectory() as tmp:
        subprocess.run([sys.executable, os.path.join(ref, "scripts/gen-fixtures.py"), "--out", tmp],
                       check=True, stdout=subprocess.DEVNULL)
        arrays, meta = {}, []
        for im in imman["image"]:
            raw = open(os.path.join(tmp, im["file"]), "rb").read()
            digest = hashlib.sha256(raw).hexdigest()
            assert digest == im["sha256"], f"{im['name']}: regenerated bytes differ from the pin"
            arrays[im["name"]] = np.frombuffer(raw, dtype=np.uint8).reshape(im["height"], im["width"])
            meta.append({"name": im["name"], "width": im["width"], "height": im["height"],
                         "sha256": digest})
    np.savez_compressed(os.path.join(HERE, "images.npz"), **arrays)
    with open(os.path.join(HERE, "images.json"), "w") as f:
        json.dump({"source": "scripts/gen-fixtures.py (fixtures/images/manifest.toml pins)",
                   "images": meta}, f, indent=1)
    print(f"wrote {len(entries)} .ifs fixtures and {len(meta)} images")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
