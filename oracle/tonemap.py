"""TEST INFRASTRUCTURE, not part of the product: f64 numpy restatement of the reference's
LDR output chain, the checker for lum_tonemap_device / lum_render_ldr.

Follows render::render (src/render.rs): auto-exposure 2594-2608 with the log-average
luminance of 525-540; the per-pixel loop 3100-3260 (vignette, white balance, hue shift,
saturation, grading, tone curve, Bayer dither, gamma_correct, brightness, contrast, sepia,
tint, colour balance, posterize); tone curves 3608-3641; gamma_correct 3648-3658; RGBA with
alpha 255 (3504).  Rust's `as u8` from f64 truncates, saturates and maps NaN to 0.

Pinned against the reference's own unit tests of these functions (src/render.rs:3665-3775):
aces(0) = 0, ACES/filmic bounded and monotone, filmic(0) ~ 0, reinhard(1) = 0.5,
linear_to_srgb(0) = 0, (1) = 255, monotone, clamps negatives.
"""
import math

import numpy as np

ACES, REINHARD, FILMIC, NONE = 0, 1, 2, 3
BAYER4 = np.array([[0, 8, 2, 10], [12, 4, 14, 6], [3, 11, 1, 9], [15, 7, 13, 5]], dtype=np.float64) / 16.0


def default_params():
    """RenderConfig defaults for the chain (src/render.rs:423-510)."""
    return dict(tone_map=ACES, auto_exposure=False, exposure=1.0, gamma=0.0, dither=False, posterize=0,
                vignette=0.0, saturation=1.0, white_balance=0.0, hue_shift=0.0, grade_shadows=(1.0, 1.0, 1.0),
                grade_highlights=(1.0, 1.0, 1.0), brightness=0.0, contrast=1.0, sepia=0.0, tint=(1.0, 1.0, 1.0),
                color_balance=(1.0, 1.0, 1.0))


def as_u8(x):
    """Rust `f64 as u8`: truncation toward zero, saturating, NaN -> 0."""
    x = np.asarray(x, dtype=np.float64)
    with np.errstate(invalid="ignore"):
        return np.where(x > 0.0, np.minimum(np.floor(x), 255.0), 0.0).astype(np.uint8)


def tone_curve(kind, x):
    x = np.fmax(np.asarray(x, dtype=np.float64), 0.0)            # f64::max ignores NaN
    if kind == REINHARD:                                            # src/render.rs:3619-3622
        return x / (1.0 + x)
    if kind == FILMIC:                                              # src/render.rs:3626-3641
        def uc2(v):
            a, b, c, d, e, f = 0.15, 0.50, 0.10, 0.20, 0.02, 0.30
            return ((v * (a * v + c * b) + d * e) / (v * (a * v + b) + d * f)) - e / f
        return np.clip(uc2(x) / uc2(11.2), 0.0, 1.0)
    if kind == NONE:
        return np.clip(x, 0.0, 1.0)
    a, b, c, d, e = 2.51, 0.03, 2.43, 0.59, 0.14                    # src/render.rs:3608-3617
    return np.clip((x * (a * x + b)) / (x * (c * x + d) + e), 0.0, 1.0)


def gamma_correct(x, gamma=0.0, dither=0.0):
    """src/render.rs:3648-3658."""
    x = np.clip(np.asarray(x, dtype=np.float64), 0.0, 1.0)
    with np.errstate(invalid="ignore"):
        if gamma > 0.0:
            s = np.power(x, 1.0 / gamma)
        else:
            s = np.where(x <= 0.0031308, 12.92 * x, 1.055 * np.power(x, 1.0 / 2.4) - 0.055)
    return as_u8(np.clip(s + dither, 0.0, 0.999) * 256.0)


def log_average_luminance(hdr):
    """src/render.rs:525-540."""
    h = np.asarray(hdr, dtype=np.float64).reshape(-1, 3)
    if len(h) == 0:
        return 0.0
    lum = 0.2126 * h[:, 0] + 0.7152 * h[:, 1] + 0.0722 * h[:, 2]
    return math.exp(float(np.log(1e-4 + np.fmax(lum, 0.0)).sum()) / len(h))


def tonemap(hdr, p=None):
    """Linear (H, W, 3) image, exposure not applied -> (H, W, 4) uint8."""
    q = default_params()
    q.update(p or {})
    hdr = np.asarray(hdr, dtype=np.float64)
    H, W = hdr.shape[:2]
    exposure = q["exposure"]
    if q["auto_exposure"]:                                           # src/render.rs:2594-2608
        la = log_average_luminance(hdr)
        exposure = (0.18 / la if la > 1e-6 else 1.0) * exposure
    jj, ii = np.meshgrid(np.arange(H, dtype=np.float64), np.arange(W, dtype=np.float64), indexing="ij")
    vf = np.ones((H, W))
    if q["vignette"] > 0.0:
        cx = (ii + 0.5) / W - 0.5
        cy = (jj + 0.5) / H - 0.5
        vf = np.fmax(1.0 - (cx * cx + cy * cy) * q["vignette"] * 4.0, 0.0)
    cr, cg, cb = (hdr[..., c] * exposure * vf for c in range(3))
    wb = q["white_balance"]
    if abs(wb) > 1e-6:
        cr, cb, cg = cr * (1.0 + wb * 0.1), cb * (1.0 - wb * 0.1), cg * (1.0 + wb * 0.02)
    if abs(q["hue_shift"]) > 1e-6:
        ang = q["hue_shift"] * (math.pi / 180.0)
        ca, sa = math.cos(ang), math.sin(ang)
        k, s3 = 1.0 / 3.0, 1.0 / math.sqrt(3.0)
        d, m, pp = ca + k * (1.0 - ca), k * (1.0 - ca) - s3 * sa, k * (1.0 - ca) + s3 * sa
        nr = cr * d + cg * m + cb * pp
        ng = cr * pp + cg * d + cb * m
        nb = cr * m + cg * pp + cb * d
        cr, cg, cb = np.fmax(nr, 0.0), np.fmax(ng, 0.0), np.fmax(nb, 0.0)
    sat = q["saturation"]
    if abs(sat - 1.0) > 1e-6:
        lum = 0.2126 * cr + 0.7152 * cg + 0.0722 * cb
        cr, cg, cb = lum + (cr - lum) * sat, lum + (cg - lum) * sat, lum + (cb - lum) * sat
    gs, gh = q["grade_shadows"], q["grade_highlights"]
    if tuple(gs) != (1.0, 1.0, 1.0) or tuple(gh) != (1.0, 1.0, 1.0):
        lum = np.fmax(0.2126 * cr + 0.7152 * cg + 0.0722 * cb, 0.0)
        t = np.clip(lum / (lum + 1.0), 0.0, 1.0)
        cr, cg, cb = (c * (gs[k] * (1.0 - t) + gh[k] * t) for k, c in enumerate((cr, cg, cb)))
    dither = (BAYER4[jj.astype(int) % 4, ii.astype(int) % 4] - 0.5) / 255.0 if q["dither"] else 0.0
    r, g, b = (gamma_correct(tone_curve(q["tone_map"], c), q["gamma"], dither).astype(np.int64) for c in (cr, cg, cb))
    br = q["brightness"]
    if abs(br) > 1e-6:
        off = int(max(min(math.trunc(br * 255.0), 32767), -32768))
        r, g, b = (np.clip(c + off, 0, 255) for c in (r, g, b))
    con = q["contrast"]
    if abs(con - 1.0) > 1e-6:
        r, g, b = (as_u8(np.clip(((c / 255.0 - 0.5) * con + 0.5) * 255.0, 0.0, 255.0)).astype(np.int64) for c in (r, g, b))
    sp = q["sepia"]
    if sp > 0.0:
        fr, fg, fb = r / 255.0, g / 255.0, b / 255.0
        sr = np.fmin(fr * 0.393 + fg * 0.769 + fb * 0.189, 1.0)
        sg = np.fmin(fr * 0.349 + fg * 0.686 + fb * 0.168, 1.0)
        sb = np.fmin(fr * 0.272 + fg * 0.534 + fb * 0.131, 1.0)
        r, g, b = (as_u8((f * (1.0 - sp) + s * sp) * 255.0).astype(np.int64) for f, s in ((fr, sr), (fg, sg), (fb, sb)))
    tint = q["tint"]
    if tint[0] < 1.0 or tint[1] < 1.0 or tint[2] < 1.0:
        r, g, b = (as_u8(np.clip((c / 255.0 * tint[k]) * 255.0, 0.0, 255.0)).astype(np.int64)
                   for k, c in enumerate((r, g, b)))
    cbal = q["color_balance"]
    if any(abs(x - 1.0) > 1e-6 for x in cbal):
        r, g, b = (as_u8(np.clip(c * cbal[k], 0.0, 255.0)).astype(np.int64) for k, c in enumerate((r, g, b)))
    if q["posterize"] >= 2:
        L = float(q["posterize"])
        # f64::round: half away from zero
        def post(c):
            x = (c / 255.0) * (L - 1.0)
            return as_u8(np.clip(np.copysign(np.floor(np.abs(x) + 0.5), x) / (L - 1.0) * 255.0, 0.0, 255.0)).astype(np.int64)
        r, g, b = post(r), post(g), post(b)
    out = np.empty((H, W, 4), dtype=np.uint8)
    out[..., 0], out[..., 1], out[..., 2], out[..., 3] = r, g, b, 255
    return out
