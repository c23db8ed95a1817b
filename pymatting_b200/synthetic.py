"""Seeded synthetic matting inputs.

The closed-form alpha path is benchmarked on generated images rather than on a
photo dataset. One generator covers every workload:

* foreground and background colour fields are random low-order 2D polynomials
  per channel plus N(0, 0.02) noise, clipped to [0, 1];
* the ground-truth alpha is a union of random ellipses, Gaussian-blurred
  (sigma 2 for the 320x240 case, 3 otherwise);
* the trimap is 1.0 where alpha > 0.99, 0.0 where alpha < 0.01 and 0.5 on the
  transition band dilated by ``band`` pixels.

Ellipses are added until the unknown fraction reaches ``unknown_fraction``;
the realised fraction is returned so callers can report it.
"""

import numpy as np
from scipy import ndimage

__all__ = ["make_matting_problem", "batch_sizes"]


def _colour_field(rng, h, w, degree=3):
    y = np.linspace(-1.0, 1.0, h)[:, None]
    x = np.linspace(-1.0, 1.0, w)[None, :]
    field = np.empty((h, w, 3))
    for c in range(3):
        f = np.zeros((h, w))
        for i in range(degree + 1):
            for j in range(degree + 1 - i):
                f = f + rng.normal() * (x ** i) * (y ** j)
        lo, hi = f.min(), f.max()
        f = (f - lo) / max(hi - lo, 1e-12)
        a = rng.uniform(0.05, 0.45)
        b = rng.uniform(0.55, 0.95)
        field[:, :, c] = a + (b - a) * f
    field += rng.normal(0.0, 0.02, size=field.shape)
    return np.clip(field, 0.0, 1.0)


def _ellipse_mask(h, w, cy, cx, ry, rx, theta):
    y0 = max(int(cy - max(ry, rx)) - 1, 0)
    y1 = min(int(cy + max(ry, rx)) + 2, h)
    x0 = max(int(cx - max(ry, rx)) - 1, 0)
    x1 = min(int(cx + max(ry, rx)) + 2, w)
    yy, xx = np.mgrid[y0:y1, x0:x1]
    dy = yy - cy
    dx = xx - cx
    ct, st = np.cos(theta), np.sin(theta)
    u = (dx * ct + dy * st) / rx
    v = (-dx * st + dy * ct) / ry
    return (y0, y1, x0, x1), (u * u + v * v) <= 1.0


def _trimap_from_alpha(alpha, band):
    fg = alpha > 0.99
    bg = alpha < 0.01
    transition = ~(fg | bg)
    if band > 0 and transition.any():
        dist = ndimage.distance_transform_edt(~transition)
        transition = dist <= band
    trimap = np.where(fg, 1.0, 0.0)
    trimap[transition] = 0.5
    return trimap


def make_matting_problem(h, w, seed, sigma=3.0, band=10, unknown_fraction=0.08,
                         dtype=np.float64):
    """Return ``(image, trimap, alpha, realised_unknown_fraction)``.

    ``image`` is ``(h, w, 3)``, ``trimap`` and ``alpha`` are ``(h, w)``, all of
    ``dtype``. The same ``(h, w, seed, ...)`` always gives the same arrays.
    """
    rng = np.random.default_rng(seed)
    fg_col = _colour_field(rng, h, w)
    bg_col = _colour_field(rng, h, w)

    # Unknown-band width per unit of ellipse perimeter: the blurred edge
    # (0.01 < alpha < 0.99 spans +-2.33 sigma) plus the dilation on each side.
    width = 2.0 * 2.33 * sigma + 2.0 * band + 1.0
    target_px = unknown_fraction * h * w
    mask = np.zeros((h, w), dtype=bool)
    est_px = 0.0
    s = min(h, w)
    # Keep one ellipse's band below ~60% of the target so small images do not
    # overshoot the requested fraction with their first ellipse.
    # Large fractions need many small ellipses: with radius ~width / fraction
    # the union covers well under half of the image when the bands add up to
    # the target, so the bands do not swallow each other.
    r_hi = min(0.32 * s, 0.6 * target_px / (2.0 * np.pi * width),
               max(1.0 * width / max(unknown_fraction, 1e-3), 4.0))
    # Every ellipse keeps a foreground interior after blur and dilation.
    r_min = 2.33 * sigma + band + 4.0
    r_hi = max(r_hi, r_min)
    r_lo = max(min(0.12 * s, 0.5 * r_hi), r_min)
    trimap = alpha = None
    realised = 0.0
    for _round in range(6):
        while est_px < target_px:
            ry = rng.uniform(r_lo, r_hi)
            rx = rng.uniform(r_lo, r_hi)
            cy = rng.uniform(0.0, 1.0) * h
            cx = rng.uniform(0.0, 1.0) * w
            theta = rng.uniform(0.0, np.pi)
            (y0, y1, x0, x1), m = _ellipse_mask(h, w, cy, cx, ry, rx, theta)
            mask[y0:y1, x0:x1] |= m
            per = np.pi * (3 * (rx + ry) - np.sqrt((3 * rx + ry) * (rx + 3 * ry)))
            est_px += per * width
        alpha = ndimage.gaussian_filter(mask.astype(np.float64), sigma)
        alpha = np.clip(alpha, 0.0, 1.0)
        trimap = _trimap_from_alpha(alpha, band)
        realised = float(np.mean(trimap == 0.5))
        if realised >= 0.85 * unknown_fraction:
            break
        # Overlapping ellipses lose band area: ask for the shortfall again.
        est_px = realised * h * w

    image = fg_col * alpha[:, :, None] + bg_col * (1.0 - alpha[:, :, None])
    image = np.clip(image, 0.0, 1.0)
    # Both constraint classes must be present (trimap_split raises otherwise).
    if not (trimap >= 0.9).any():
        trimap[h // 2, w // 2] = 1.0
    if not (trimap <= 0.1).any():
        trimap[0, 0] = 0.0
    return (image.astype(dtype), trimap.astype(dtype), alpha.astype(dtype),
            realised)


# Image sizes of the mixed-size batch workload (h, w).
BATCH_SIZES = [(256, 256), (480, 640), (768, 1024), (720, 1280), (1080, 1920),
               (1536, 2048)]


def batch_sizes(count, seed):
    """Sizes and unknown fractions for a mixed batch: ``[(h, w, frac, seed_k)]``."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        h, w = BATCH_SIZES[int(rng.integers(0, len(BATCH_SIZES)))]
        frac = float(rng.uniform(0.05, 0.25))
        out.append((h, w, frac, seed + 1 + k))
    return out
