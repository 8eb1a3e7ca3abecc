"""Seeded synthetic RAW scenes for the develop path.

There is no public dataset and no RAW fixture for this path, so benchmarks and
parity tests run on seeded synthetic scenes with the shapes, CFA layouts and
value ranges of the workloads libraw_enhanced develops:

* ``scene_rgb(h, w, seed)``: 64 rotated rectangles (centre uniform in the
  frame, sides uniform in [0.03, 0.35] * min(h, w), angle uniform in [0, pi),
  RGB uniform in [0.02, 0.9]) over a seeded background, plus 2-octave value
  noise (lattices of 64 and 32 px, smoothstep interpolation, amplitude 0.05)
  and one 256x256 zone plate ``0.5 + 0.4 cos(pi r^2 / 256)``.
* ``mosaic(rgb, cfa)``: sample the scene through a Bayer (LibRaw ``filters``
  bit pattern) or a 6x6 X-Trans CFA, add Poisson-Gaussian noise
  ``Poisson(4000 x) / 4000 + N(0, 0.002^2)`` and multiply by the per-site
  white-balance gain.
* ``bayer_51mp_fringed``: the 8736x5856 develop workload: a 1536x1024 scene
  upscaled bilinearly, with purple fringing injected (R and B blurred with
  sigma 2 px where Sobel(luma) is high and luma > 0.8), clipped at 1.0, then
  mosaiced RGGB with WB (2, 1, 1.5, 1).
* ``xtrans_lateral_ca``: the 6240x4160 X-Trans workload with radial lateral
  CA (R scaled by 1.0008, B by 0.9992 about the centre) before mosaicing.

Every generator is deterministic for a given seed (numpy PCG64).
"""
from __future__ import annotations

import numpy as np

# LibRaw `filters` words for the four Bayer layouts (core/metal/shader_common.h
# fcol_bayer_native: filters >> (((row << 1 & 14) | (col & 1)) << 1) & 3).
FILTERS = {
    "RGGB": 0x94949494,
    "BGGR": 0x16161616,
    "GRBG": 0x61616161,
    "GBRG": 0x49494949,
}
FILTERS_XTRANS = 9

# The standard Fujifilm X-Trans 6x6 layout (0 = R, 1 = G, 2 = B):
# 20 green, 8 red and 8 blue sites per period.
XTRANS_STD = np.array(
    [
        [1, 1, 0, 1, 1, 2],
        [1, 1, 2, 1, 1, 0],
        [2, 0, 1, 0, 2, 1],
        [1, 1, 2, 1, 1, 0],
        [1, 1, 0, 1, 1, 2],
        [0, 2, 1, 2, 0, 1],
    ],
    dtype=np.int8,
)


def fcol_bayer_native(row, col, filters: int):
    """CFA colour index 0..3 (3 = second green) at (row, col)."""
    row = np.asarray(row, dtype=np.int64)
    col = np.asarray(col, dtype=np.int64)
    return (int(filters) >> ((((row << 1) & 14) | (col & 1)) << 1)) & 3


def cfa_map(h: int, w: int, cfa) -> np.ndarray:
    """Per-pixel native colour index (0..3 for Bayer, 0..2 for X-Trans)."""
    if isinstance(cfa, np.ndarray):
        rows = np.arange(h)[:, None] % 6
        cols = np.arange(w)[None, :] % 6
        return np.asarray(cfa, dtype=np.int64)[rows, cols]
    filters = FILTERS[cfa] if isinstance(cfa, str) else int(cfa)
    rows = np.arange(h)[:, None]
    cols = np.arange(w)[None, :]
    return fcol_bayer_native(rows, cols, filters)


def _value_noise(h, w, cell, rng):
    gh, gw = h // cell + 2, w // cell + 2
    lat = rng.uniform(-1.0, 1.0, size=(gh, gw)).astype(np.float32)
    y = np.arange(h, dtype=np.float32) / cell
    x = np.arange(w, dtype=np.float32) / cell
    y0 = np.floor(y).astype(np.int64)
    x0 = np.floor(x).astype(np.int64)
    ty = y - y0
    tx = x - x0
    ty = ty * ty * (3 - 2 * ty)
    tx = tx * tx * (3 - 2 * tx)
    a = lat[y0][:, x0]
    b = lat[y0][:, x0 + 1]
    c = lat[y0 + 1][:, x0]
    d = lat[y0 + 1][:, x0 + 1]
    top = a + (b - a) * tx[None, :]
    bot = c + (d - c) * tx[None, :]
    return top + (bot - top) * ty[:, None]


def scene_rgb(h: int, w: int, seed: int, n_rects: int = 64) -> np.ndarray:
    """Linear RGB scene in [0, ~1], float32 (h, w, 3)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    img = np.empty((h, w, 3), dtype=np.float32)
    img[...] = rng.uniform(0.02, 0.9, size=3).astype(np.float32)
    m = min(h, w)
    for _ in range(n_rects):
        cy, cx = rng.uniform(0, h), rng.uniform(0, w)
        sa, sb = rng.uniform(0.03, 0.35, size=2) * m
        th = rng.uniform(0, np.pi)
        col = rng.uniform(0.02, 0.9, size=3).astype(np.float32)
        rad = 0.5 * np.hypot(sa, sb)
        y0, y1 = max(0, int(cy - rad)), min(h, int(cy + rad) + 1)
        x0, x1 = max(0, int(cx - rad)), min(w, int(cx + rad) + 1)
        if y0 >= y1 or x0 >= x1:
            continue
        yy = np.arange(y0, y1, dtype=np.float32)[:, None] - cy
        xx = np.arange(x0, x1, dtype=np.float32)[None, :] - cx
        c, s = np.cos(th), np.sin(th)
        u = c * xx + s * yy
        v = -s * xx + c * yy
        inside = (np.abs(u) <= 0.5 * sa) & (np.abs(v) <= 0.5 * sb)
        img[y0:y1, x0:x1][inside] = col
    noise = 0.05 * (_value_noise(h, w, 64, rng) + 0.5 * _value_noise(h, w, 32, rng)) / 1.5
    img += noise[:, :, None]
    # zone plate
    zs = min(256, h, w)
    zy = int(rng.integers(0, h - zs + 1))
    zx = int(rng.integers(0, w - zs + 1))
    r = np.arange(zs, dtype=np.float32) - zs / 2
    r2 = r[:, None] ** 2 + r[None, :] ** 2
    zp = 0.5 + 0.4 * np.cos(np.pi * r2 / 256.0)
    img[zy : zy + zs, zx : zx + zs] = zp[:, :, None].astype(np.float32)
    np.clip(img, 0.0, None, out=img)
    return img


def mosaic(rgb: np.ndarray, cfa, wb, seed: int, noise: bool = True) -> np.ndarray:
    """Dense float32 (h, w) CFA mosaic with Poisson-Gaussian noise and WB.

    ``wb`` holds 4 gains indexed by the native colour (R, G, B, G2).
    """
    h, w, _ = rgb.shape
    idx = cfa_map(h, w, cfa)
    ch = np.where(idx == 3, 1, idx)
    x = np.take_along_axis(rgb, ch[:, :, None], axis=2)[:, :, 0].astype(np.float32)
    if noise:
        rng = np.random.Generator(np.random.PCG64(seed + 7919))
        x = rng.poisson(np.clip(x, 0, None) * 4000.0).astype(np.float32) / 4000.0
        x += rng.normal(0.0, 0.002, size=x.shape).astype(np.float32)
        np.clip(x, 0.0, None, out=x)
    gains = np.asarray(wb, dtype=np.float32)[idx]
    return (x * gains).astype(np.float32)


def sparse_rgb(mos: np.ndarray, cfa) -> np.ndarray:
    """The reference's raw-buffer layout: (h, w, 3) float32 with only the
    native channel of each site set (G2 stored in channel 1), zeros elsewhere."""
    h, w = mos.shape
    idx = cfa_map(h, w, cfa)
    ch = np.where(idx == 3, 1, idx)
    out = np.zeros((h, w, 3), dtype=np.float32)
    np.put_along_axis(out, ch[:, :, None], mos[:, :, None], axis=2)
    return out


def _resize_bilinear(img: np.ndarray, h: int, w: int) -> np.ndarray:
    sh, sw = img.shape[:2]
    ys = (np.arange(h, dtype=np.float32) + 0.5) * (sh / h) - 0.5
    xs = (np.arange(w, dtype=np.float32) + 0.5) * (sw / w) - 0.5
    ys = np.clip(ys, 0, sh - 1)
    xs = np.clip(xs, 0, sw - 1)
    y0 = np.minimum(np.floor(ys).astype(np.int64), sh - 2)
    x0 = np.minimum(np.floor(xs).astype(np.int64), sw - 2)
    fy = (ys - y0)[:, None, None]
    fx = (xs - x0)[None, :, None]
    out = np.empty((h, w, img.shape[2]), dtype=np.float32)
    # process in row blocks to bound temporaries
    for r0 in range(0, h, 1024):
        r1 = min(h, r0 + 1024)
        a = img[y0[r0:r1]][:, x0]
        b = img[y0[r0:r1]][:, x0 + 1]
        c = img[y0[r0:r1] + 1][:, x0]
        d = img[y0[r0:r1] + 1][:, x0 + 1]
        fyb = fy[r0:r1]
        top = a + (b - a) * fx
        bot = c + (d - c) * fx
        out[r0:r1] = top + (bot - top) * fyb
    return out


def inject_fringing(rgb: np.ndarray, sigma: float = 2.0) -> np.ndarray:
    """Blur R and B (sigma px) where Sobel(luma) is high and luma > 0.8."""
    from scipy import ndimage

    luma = 0.2126 * rgb[:, :, 0] + 0.7152 * rgb[:, :, 1] + 0.0722 * rgb[:, :, 2]
    gx = ndimage.sobel(luma, axis=1)
    gy = ndimage.sobel(luma, axis=0)
    mag = np.hypot(gx, gy)
    edge = (mag > 0.25) & (ndimage.maximum_filter(luma, size=5) > 0.8)
    wmask = ndimage.gaussian_filter(edge.astype(np.float32), 1.5)
    wmask = np.clip(wmask * 2.0, 0.0, 1.0)
    out = rgb.copy()
    for c in (0, 2):
        blurred = ndimage.gaussian_filter(rgb[:, :, c], sigma)
        out[:, :, c] = rgb[:, :, c] + (blurred - rgb[:, :, c]) * wmask
    return out


def bayer_scene(h: int, w: int, seed: int, cfa="RGGB", wb=(2.0, 1.0, 1.5, 1.0)) -> np.ndarray:
    """Dense Bayer mosaic of a native-resolution scene (small/medium sizes)."""
    return mosaic(scene_rgb(h, w, seed), cfa, wb, seed)


def bayer_51mp_fringed(seed: int = 2, h: int = 5856, w: int = 8736, base=(1024, 1536)) -> np.ndarray:
    """The 51 MP fringed RGGB develop workload (dense float32 mosaic)."""
    small = scene_rgb(base[0], base[1], seed)
    big = _resize_bilinear(small, h, w)
    big = inject_fringing(big, 2.0)
    np.clip(big, 0.0, 1.0, out=big)
    return mosaic(big, "RGGB", (2.0, 1.0, 1.5, 1.0), seed)


def radial_ca(rgb: np.ndarray, r_scale=1.0008, b_scale=0.9992) -> np.ndarray:
    """Scale R and B about the image centre (bilinear, clamp to edge)."""
    h, w, _ = rgb.shape
    cy, cx = (h - 1) / 2.0, (w - 1) / 2.0
    out = rgb.copy()
    yy = np.arange(h, dtype=np.float32)[:, None]
    xx = np.arange(w, dtype=np.float32)[None, :]
    for c, s in ((0, r_scale), (2, b_scale)):
        sy = np.clip(cy + (yy - cy) / s, 0, h - 1)
        sx = np.clip(cx + (xx - cx) / s, 0, w - 1)
        y0 = np.minimum(np.floor(sy).astype(np.int64), h - 2)
        x0 = np.minimum(np.floor(sx).astype(np.int64), w - 2)
        fy = sy - y0
        fx = sx - x0
        p = rgb[:, :, c]
        top = p[y0, x0] * (1 - fx) + p[y0, x0 + 1] * fx
        bot = p[y0 + 1, x0] * (1 - fx) + p[y0 + 1, x0 + 1] * fx
        out[:, :, c] = top * (1 - fy) + bot * fy
    return out


def xtrans_lateral_ca(seed: int = 3, h: int = 4160, w: int = 6240, wb=(1.8, 1.0, 1.6, 1.0)) -> np.ndarray:
    """The X-Trans workload with radial lateral CA (dense float32 mosaic)."""
    rgb = radial_ca(scene_rgb(h, w, seed))
    return mosaic(rgb, XTRANS_STD, wb, seed)


def random_cfa_name(rng) -> str:
    return ["RGGB", "BGGR", "GRBG", "GBRG"][int(rng.integers(0, 4))]


# ------------------------------------------------------------ multi-image sets
BATCH_SIZES = [(3024, 4032), (4000, 6000), (5504, 8256), (6336, 9504)]


def batch_specs(n: int = 32, seed_base: int = 100):
    """The batched-develop set: per image (seed, h, w, cfa, wb), drawn by seed
    from the four sensor sizes and four Bayer layouts, WB R ~ U[1.5, 2.5],
    B ~ U[1.2, 2.0], G = 1."""
    out = []
    for i in range(n):
        rng = np.random.Generator(np.random.PCG64(seed_base + i))
        h, w = BATCH_SIZES[int(rng.integers(0, 4))]
        cfa = random_cfa_name(rng)
        wb = (float(rng.uniform(1.5, 2.5)), 1.0, float(rng.uniform(1.2, 2.0)), 1.0)
        out.append((seed_base + i, h, w, cfa, wb))
    return out


def mosaic_upscaled_torch(seed: int, h: int, w: int, cfa, wb, base=(512, 768), device="cuda"):
    """A large seeded mosaic generated on the GPU (for multi-image benchmarks
    where numpy generation would take minutes): the seeded scene at `base`
    resolution, upscaled bilinearly, mosaiced through `cfa` (Bayer name or a
    6x6 X-Trans pattern), Poisson-Gaussian noise (gain 1/4000, read sigma
    0.002) and per-site WB.  Returns a float32 CUDA tensor (h, w)."""
    import torch
    import torch.nn.functional as F

    small = torch.from_numpy(scene_rgb(base[0], base[1], seed)).to(device)
    big = F.interpolate(small.permute(2, 0, 1)[None], size=(h, w), mode="bilinear", align_corners=False)[0]
    period = 6 if isinstance(cfa, np.ndarray) else 2
    idx = torch.from_numpy(cfa_map(period, period, cfa)).to(device)
    ii = idx.repeat((h + period - 1) // period, (w + period - 1) // period)[:h, :w]
    ch = torch.where(ii == 3, torch.ones_like(ii), ii)
    x = torch.gather(big, 0, ch[None]).squeeze(0).clamp_min_(0)
    g = torch.Generator(device=device)
    g.manual_seed(seed + 7919)
    x = torch.poisson(x * 4000.0, generator=g) / 4000.0
    x += torch.randn(x.shape, generator=g, device=device) * 0.002
    x.clamp_min_(0)
    gains = torch.tensor(list(wb), dtype=torch.float32, device=device)[ii]
    return (x * gains).float().contiguous()


def xtrans_lateral_ca_torch(seed: int = 3, h: int = 4160, w: int = 6240, wb=(1.8, 1.0, 1.6, 1.0),
                            r_scale=1.0008, b_scale=0.9992, base=(1024, 1536), device="cuda"):
    """The X-Trans lateral-CA workload generated on the GPU: the seeded scene
    at `base` resolution upscaled bilinearly, R and B scaled radially about
    the image centre (bilinear, clamp to edge), mosaiced through the standard
    6x6 X-Trans CFA with Poisson-Gaussian noise and WB.  float32 CUDA (h, w)."""
    import torch
    import torch.nn.functional as F

    small = torch.from_numpy(scene_rgb(base[0], base[1], seed)).to(device)
    big = F.interpolate(small.permute(2, 0, 1)[None], size=(h, w), mode="bilinear", align_corners=False)[0]
    cy, cx = (h - 1) / 2.0, (w - 1) / 2.0
    yy = torch.arange(h, device=device, dtype=torch.float32)[:, None]
    xx = torch.arange(w, device=device, dtype=torch.float32)[None, :]
    for c, s in ((0, r_scale), (2, b_scale)):
        sy = (cy + (yy - cy) / s).expand(h, w)
        sx = (cx + (xx - cx) / s).expand(h, w)
        grid = torch.stack([sx / (w - 1) * 2 - 1, sy / (h - 1) * 2 - 1], dim=-1)[None]
        big[c] = F.grid_sample(big[c][None, None], grid, mode="bilinear", padding_mode="border",
                               align_corners=True)[0, 0]
    idx = torch.from_numpy(cfa_map(6, 6, XTRANS_STD)).to(device)
    ii = idx.repeat((h + 5) // 6, (w + 5) // 6)[:h, :w]
    x = torch.gather(big, 0, ii[None]).squeeze(0).clamp_min_(0)
    g = torch.Generator(device=device)
    g.manual_seed(seed + 7919)
    x = torch.poisson(x * 4000.0, generator=g) / 4000.0
    x += torch.randn(x.shape, generator=g, device=device) * 0.002
    x.clamp_min_(0)
    gains = torch.tensor(list(wb), dtype=torch.float32, device=device)[ii]
    return (x * gains).float().contiguous()
