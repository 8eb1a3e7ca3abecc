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
