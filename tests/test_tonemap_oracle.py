"""The LDR chain's oracle (oracle/tonemap.py) pinned by the reference's own unit tests of the
tone curves and the sRGB transfer (src/render.rs:3665-3775), plus the scene-file mapping."""
import numpy as np
import pytest

from luminara_b200 import abi
from luminara_b200.toml_scene import UnsupportedSceneError, load_scene, tonemap_config
from oracle import tonemap as OT


def test_tone_curves_known_answers():
    assert OT.tone_curve(OT.ACES, 0.0) == 0.0
    x = np.arange(100) * 0.5
    for kind in (OT.ACES, OT.FILMIC):
        y = OT.tone_curve(kind, x)
        assert ((y >= 0) & (y <= 1)).all()
        assert (np.diff(OT.tone_curve(kind, np.arange(1, 100) * 0.1)) >= 0).all()
    assert abs(OT.tone_curve(OT.FILMIC, 0.0)) < 0.01
    assert OT.tone_curve(OT.REINHARD, 0.0) == 0.0 and abs(OT.tone_curve(OT.REINHARD, 1.0) - 0.5) < 1e-6
    assert (np.diff(OT.tone_curve(OT.REINHARD, np.arange(1, 50.0))) > 0).all()


def test_srgb_known_answers():
    assert OT.gamma_correct(0.0) == 0 and OT.gamma_correct(1.0) == 255 and OT.gamma_correct(-1.0) == 0
    y = OT.gamma_correct(np.linspace(0, 1, 1001))
    assert (np.diff(y.astype(int)) >= 0).all()
    assert OT.gamma_correct(np.nan) == 0
    assert OT.gamma_correct(0.25, gamma=2.0) == int(0.5 * 256)


def test_chain_defaults_and_auto_exposure():
    hdr = np.full((2, 3, 3), 0.18)
    out = OT.tonemap(hdr, {"auto_exposure": True, "tone_map": OT.NONE})
    # log-average of 0.18 (+1e-4 inside the log) maps to ~0.18 after the key value
    assert out.shape == (2, 3, 4) and (out[..., 3] == 255).all()
    assert abs(int(out[0, 0, 0]) - int(OT.gamma_correct(0.18 * 0.18 / (0.18 + 1e-4)))) <= 1


def test_scene_file_chain_settings():
    cfg, world, post = load_scene('[render]\ntone_map = "filmic"\ngamma = 2.2\ndither = true\nvignette = 0.3\n'
                                  'saturation = 1.2\ngrade_shadows = [0.9, 1.0, 1.1]\nposterize = 8\nexposure = 2.0\n'
                                  'solarize = -1.0\ndenoise = false\n'
                                  '[[sphere]]\ncenter = [0, 0, 0]\nradius = 1\nmaterial = { type = "glass" }\n')
    tm = tonemap_config(post)
    assert cfg.exposure == 2.0
    assert (tm.tone_map, tm.gamma, tm.dither, tm.vignette, tm.saturation, tm.posterize) == \
        (abi.TONEMAP_FILMIC, 2.2, True, 0.3, 1.2, 8)
    assert tm.grade_shadows == (0.9, 1.0, 1.1)
    assert tonemap_config({"tone_map": "something"}).tone_map == abi.TONEMAP_ACES
    with pytest.raises(UnsupportedSceneError) as e:
        tonemap_config({"bloom": 0.3, "sharpen": 0.0, "blur": 2.0})
    assert e.value.items == ["render.bloom", "render.blur"]
