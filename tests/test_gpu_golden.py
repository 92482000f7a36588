"""The device against the committed golden frames of the keyed oracle
(tests/golden/keyed_renders.npz): the keyed-render tolerance of the live oracle comparisons
(a fraction of pixels within 2e-3 * (1 + |ref|) per channel, image means within 0.5%) and the
same path count."""
import json
import os

import numpy as np
import pytest

import luminara_b200 as L
from tests.golden import make_golden as G

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "keyed_renders.npz")
_z = np.load(FIXTURE)
KEYED = [e for e in json.loads(bytes(_z["manifest"]).decode()) if e["mode"] == "keyed"]


@pytest.mark.parametrize("entry", KEYED, ids=[e["name"] for e in KEYED])
def test_device_matches_golden_frame(entry):
    ref = np.load(FIXTURE)[entry["name"]].astype(np.float64)
    world, cfg = G.scene(entry["workload"], entry["kw"])
    img, st = L.GpuScene(world).render(cfg)
    close = np.abs(img - ref) <= 2e-3 * (1.0 + np.abs(ref))
    assert close.all(axis=2).mean() >= entry["frac"], f"only {close.all(axis=2).mean():.4f} of pixels match"
    m_g, m_r = img.mean(axis=(0, 1)), ref.mean(axis=(0, 1))
    assert np.all(np.abs(m_g - m_r) <= 5e-3 * np.maximum(m_r, 1e-3)), (m_g, m_r)
    assert st.paths == entry["paths"] and st.error_flags == 0
