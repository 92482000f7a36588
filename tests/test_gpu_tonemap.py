"""GPU tests of the LDR colour chain (lum_tonemap_device, lum_render_ldr) against the f64 oracle.

The device computes the chain in f64 without FMA contraction, so bytes equal the oracle's
except where a last-bit difference of pow/log/exp (CUDA's versus the host's) lands on a
quantisation boundary: >= 99.99% of channel bytes identical and no byte off by more than 1.
"""
import numpy as np
import pytest

import luminara_b200 as L
from luminara_b200 import abi
from luminara_b200 import workloads as W
from oracle import tonemap as OT

pytestmark = pytest.mark.gpu

CHAINS = [
    {},
    {"tone_map": OT.REINHARD, "gamma": 2.2, "dither": True, "vignette": 0.4, "exposure": 1.7},
    {"tone_map": OT.FILMIC, "auto_exposure": True, "saturation": 1.3, "white_balance": 0.5, "hue_shift": 25.0,
     "grade_shadows": (0.9, 1.0, 1.15), "grade_highlights": (1.1, 1.0, 0.9)},
    {"tone_map": OT.NONE, "brightness": 0.05, "contrast": 1.4, "sepia": 0.3, "tint": (1.0, 0.9, 0.8),
     "color_balance": (1.1, 1.0, 0.95), "posterize": 6},
    {"auto_exposure": True, "exposure": 0.5, "dither": True, "hue_shift": -40.0, "saturation": 0.6},
]


def tm_config(d):
    tm = L.ToneMapConfig()
    for k, v in d.items():
        setattr(tm, k, v)
    return tm


def compare(got, want):
    diff = np.abs(got.astype(int) - want.astype(int))
    assert diff.max() <= 1, diff.max()
    assert (diff == 0).mean() >= 0.9999, (diff == 0).mean()


def hdr_image(h, w, seed=0):
    rng = np.random.default_rng(seed)
    img = np.exp(rng.normal(-1.0, 1.5, (h, w, 3))).astype(np.float32)        # 5 decades of radiance
    img[rng.random((h, w)) < 0.02] = 0.0
    img[0, 0] = (-0.5, 2.0, 1e4)
    return img


@pytest.mark.parametrize("chain", range(len(CHAINS)))
@pytest.mark.parametrize("shape", [(135, 240), (23, 37)])
def test_tonemap_device_matches_oracle(chain, shape):
    import torch
    h, w = shape
    img = hdr_image(h, w, chain)
    d_hdr = torch.from_numpy(img).cuda()
    d_out = torch.empty((h, w, 4), dtype=torch.uint8, device="cuda")
    scratch = torch.empty(abi.TONEMAP_SCRATCH_BYTES, dtype=torch.uint8, device="cuda")
    L.tonemap_device(d_hdr.data_ptr(), w, h, tm_config(CHAINS[chain]), scratch.data_ptr(), d_out.data_ptr())
    torch.cuda.synchronize()
    compare(d_out.cpu().numpy(), OT.tonemap(img, CHAINS[chain]))


def test_unaligned_buffers_take_the_scalar_path():
    import torch
    h, w = 31, 17
    img = hdr_image(h, w, 5)
    flat = torch.zeros(h * w * 3 + 1, dtype=torch.float32, device="cuda")
    flat[1:] = torch.from_numpy(img).reshape(-1).cuda()
    out = torch.zeros(h * w * 4 + 3, dtype=torch.uint8, device="cuda")
    L.tonemap_device(flat.data_ptr() + 4, w, h, tm_config(CHAINS[1]), 0, out.data_ptr() + 3)
    torch.cuda.synchronize()
    compare(out[3:].cpu().numpy().reshape(h, w, 4), OT.tonemap(img, CHAINS[1]))


def test_auto_exposure_needs_scratch_and_bad_tone_map_is_rejected():
    import torch
    d = torch.ones((4, 4, 3), dtype=torch.float32, device="cuda")
    o = torch.empty((4, 4, 4), dtype=torch.uint8, device="cuda")
    with pytest.raises(L.LuminaraError):
        L.tonemap_device(d.data_ptr(), 4, 4, tm_config({"auto_exposure": True}), 0, o.data_ptr())
    with pytest.raises(L.LuminaraError):
        L.tonemap_device(d.data_ptr(), 4, 4, tm_config({"tone_map": 7}), 0, o.data_ptr())


@pytest.mark.parametrize("chain", [0, 2, 3])
def test_render_ldr_is_the_chain_over_the_hdr_render(chain):
    world, cfg = W.box_room(width=96, height=64, spp=16)
    world.camera.aspect_ratio = 96 / 64
    cfg.exposure = 1.5
    sc = L.GpuScene(world)
    ldr, st = sc.render_ldr(cfg, tm_config(CHAINS[chain]))
    assert st.paths == 96 * 64 * 16 and ldr.shape == (64, 96, 4)
    cfg1 = L.RenderConfig(**{**cfg.__dict__, "exposure": 1.0})
    hdr, _ = sc.render(cfg1)
    want = OT.tonemap(hdr, {**CHAINS[chain], "exposure": 1.5})       # the render's exposure, not tm's
    compare(ldr, want)
    assert ldr[..., :3].max() > 100


@pytest.mark.parametrize("exposure", [1.0, 4.0, 0.25, 2.0 ** -20])
def test_power_of_two_exposure_integer_keys(exposure):
    """An exposure 2^k takes the byte table with keys formed from the f32 bits (x = v * 2^k is
    exact); zero, negative, NaN, denormal and very large values fall back to the f64 key.  The
    bytes must be the chain's over eight decades and at those edges."""
    import torch
    rng = np.random.default_rng(7)
    h, w = 64, 256
    img = np.exp(rng.uniform(-12.0, 12.0, (h, w, 3))).astype(np.float32)
    edges = np.array([np.nan, 0.0, -0.0, -1.0, 1e-45, 1e-39, 1.17e-38, 2.0 ** 99, 6.4e29, 1e30, 1e35, 3e38],
                     dtype=np.float32)
    img.reshape(-1)[: edges.size] = edges
    d_hdr = torch.from_numpy(img).cuda()
    d_out = torch.empty((h, w, 4), dtype=torch.uint8, device="cuda")
    scratch = torch.empty(abi.TONEMAP_SCRATCH_BYTES, dtype=torch.uint8, device="cuda")
    L.tonemap_device(d_hdr.data_ptr(), w, h, tm_config({"exposure": exposure}), scratch.data_ptr(), d_out.data_ptr())
    torch.cuda.synchronize()
    got = d_out.cpu().numpy()
    want = OT.tonemap(img, {"exposure": exposure})
    compare(got, want)
    np.testing.assert_array_equal(got.reshape(-1, 4)[:4, :3].reshape(-1), want.reshape(-1, 4)[:4, :3].reshape(-1))
