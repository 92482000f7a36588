"""Writes tests/golden/keyed_renders.npz: small seeded frames rendered by the oracle.

The reference (a Rust crate) cannot be built here and ships no golden images, so these
fixtures are the oracle's own output: the keyed estimator (the device's random-number mapping,
evaluated in f64) and the stream estimator (the reference's per-row generator), on the
workloads' scenes at sizes the oracle renders in well under a second.  The oracle itself is
pinned to the reference's unit-test known answers (tests/test_oracle_kat.py); these frames pin
its whole-image output against regressions, and the GPU tests compare the device with them.

Run from the repository root:  python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from luminara_b200 import workloads as W  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "keyed_renders.npz")

# (name, workload, keyword arguments, mode, fraction of pixels the device must match)
CASES = [
    ("box_room_keyed", "box_room", dict(width=48, height=48, spp=4), "keyed", 0.97),
    ("random_spheres_keyed", "random_spheres", dict(width=64, height=36, spp=4), "keyed", 0.97),
    ("diff_quads_keyed", "diff_quads", dict(width=48, height=48, spp=4), "keyed", 0.97),
    ("material_zoo_keyed", "material_zoo", dict(width=96, height=72, spp=4), "keyed", 0.95),
    ("box_room_stream", "box_room", dict(width=16, height=16, spp=4), "stream", None),
]


def scene(workload, kw):
    """The workload's world and config at the fixture's size (camera aspect follows the frame)."""
    world, cfg = W.CONFIGS[workload]()
    cfg.width, cfg.height, cfg.samples_per_pixel = kw["width"], kw["height"], kw["spp"]
    world.camera.aspect_ratio = kw["width"] / kw["height"]
    return world, cfg


def render(workload, kw, mode):
    world, cfg = scene(workload, kw)
    img, st = O.OracleScene(world).render(cfg, mode=O.MODE_KEYED if mode == "keyed" else O.MODE_STREAM)
    return img, st


def main():
    arrays, manifest = {}, []
    for name, workload, kw, mode, frac in CASES:
        img, st = render(workload, kw, mode)
        arrays[name] = img.astype(np.float32)
        manifest.append({"name": name, "workload": workload, "kw": kw, "mode": mode, "frac": frac,
                         "paths": int(st.paths), "segments": int(st.segments)})
    arrays["manifest"] = np.frombuffer(json.dumps(manifest).encode(), dtype=np.uint8)
    np.savez_compressed(OUT, **arrays)
    print(f"wrote {OUT}: {', '.join(c[0] for c in CASES)}")


if __name__ == "__main__":
    main()
