"""The oracle against the committed golden frames (tests/golden/keyed_renders.npz, written by
tests/golden/make_golden.py): keyed and stream renders of small seeded frames must come out
the same, rounded to f32, with the same path and segment counts."""
import json
import os

import numpy as np
import pytest

from tests.golden import make_golden as G

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "keyed_renders.npz")


def load():
    z = np.load(FIXTURE)
    return z, json.loads(bytes(z["manifest"]).decode())


_, MANIFEST = load()


@pytest.mark.parametrize("entry", MANIFEST, ids=[e["name"] for e in MANIFEST])
def test_oracle_reproduces_golden_frame(entry):
    z, _ = load()
    img, st = G.render(entry["workload"], entry["kw"], entry["mode"])
    gold = z[entry["name"]]
    assert img.shape == gold.shape
    np.testing.assert_allclose(img.astype(np.float32), gold, rtol=1e-6, atol=1e-7)
    assert st.paths == entry["paths"] and st.segments == entry["segments"]
