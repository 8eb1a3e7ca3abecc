"""Shared helpers for the parity tests: error metrics with the acceptance
tolerances (max-abs <= 1e-4 on the [0,1] scale, PSNR >= 90 dB at peak 1.0)."""
import numpy as np

MAX_ABS = 1e-4
MIN_PSNR = 90.0


def psnr(a, b, peak=1.0):
    d = np.asarray(a, np.float64) - np.asarray(b, np.float64)
    mse = float(np.mean(d * d))
    if mse == 0.0:
        return float("inf")
    return 10.0 * np.log10(peak * peak / mse)


def report(a, b, mask=None):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if mask is not None:
        a = a[mask]
        b = b[mask]
    d = np.abs(a - b)
    return {
        "max_abs": float(d.max()) if d.size else 0.0,
        "psnr": psnr(a, b),
        "n_over": int((d > MAX_ABS).sum()),
        "n": int(d.size),
    }


def assert_parity(gpu, ref, mask=None, max_abs=MAX_ABS, min_psnr=MIN_PSNR, what=""):
    r = report(gpu, ref, mask)
    assert r["max_abs"] <= max_abs and r["psnr"] >= min_psnr, f"{what} parity failed: {r}"
    return r


def frame_mask(h, w, band):
    """True away from a `band`-px frame (for reporting edge bands separately)."""
    m = np.zeros((h, w), bool)
    m[band : h - band, band : w - band] = True
    return m


def amaze_stale_mask(h, w):
    """Pixels whose reference AMaZE value depends on per-thread scratch.

    The reference never fills the 16x16 apron corners of the tiles that touch
    two image edges (core/cpu_accelerator.cpp:1326), so those cells hold what
    the OpenMP thread's previous tile left there.  Their influence reaches (a)
    the outputs next to each image corner and (b), through pmwt being stored
    half-indexed over dirwts1 (:1507) and dirwts1 being read full-indexed in
    stage 9 (:1556), a band of tile rows near rrmax/2 in the two bottom corner
    tiles.  Returns True on those pixels; parity there is reported, not
    asserted, because the reference itself varies with the thread split.
    """
    TS = 160
    m = np.zeros((h, w), bool)
    for top in range(-16, h, TS - 32):
        for left in range(-16, w, TS - 32):
            bottom, right = min(top + TS, h + 16), min(left + TS, w + 16)
            rr1, cc1 = bottom - top, right - left
            rows, cols = [], []
            if top < 0:
                rows.append((0, 16))
            if bottom > h:
                rrmax = h - top
                rows.append((rrmax, min(rrmax + 16, rr1)))
            if left < 0:
                cols.append((0, 16))
            if right > w:
                ccmax = w - left
                cols.append((ccmax, min(ccmax + 16, cc1)))
            for r0, r1 in rows:
                for c0, c1 in cols:
                    # outputs next to the unfilled corner cells
                    y0, y1 = max(0, top + r0 - 20), min(h, top + r1 + 20)
                    x0, x1 = max(0, left + c0 - 20), min(w, left + c1 + 20)
                    m[y0:y1, x0:x1] = True
                    if r0 == 0:
                        continue  # top corners never reach stage 9's dirwts1 rows
                    # pmwt rows r0-2 .. min(r1, rr1-8)+2 land on dirwts1 rows /2
                    a0 = max(0, (r0 - 3) // 2 - 6)
                    a1 = (min(r1, rr1 - 8) + 2) // 2 + 6
                    p0, p1 = max(0, c0 // 2 - 3), (c1 + 1) // 2 + 3
                    for base in (0, TS // 2):
                        xx0, xx1 = max(0, left + base + p0 - 6), min(w, left + base + p1 + 6)
                        m[max(0, top + a0) : min(h, top + a1), xx0:xx1] = True
    return m


def dilate(mask, r):
    """Binary dilation by a (2r+1)^2 square (numpy only)."""
    out = mask.copy()
    h, w = mask.shape
    ys, xs = np.nonzero(mask)
    for y, x in zip(ys, xs):
        out[max(0, y - r) : y + r + 1, max(0, x - r) : x + r + 1] = True
    return out
