"""Rate-distortion helpers: PSNR and the Bjontegaard delta rate.

BD-rate (G. Bjontegaard, "Calculation of average PSNR differences between
RD-curves", VCEG-M33, 2001): for each codec fit log(rate) as a cubic
polynomial of PSNR through its RD points, integrate both fits over the PSNR
interval the two curves share, and turn the mean log-rate difference into a
percentage. Positive = the test codec needs more bits than the anchor for the
same quality.
"""
import numpy as np


def psnr(a, b, peak=255.0):
    """PSNR in dB between two uint8 arrays (inf for identical inputs)."""
    d = a.astype(np.float64) - b.astype(np.float64)
    mse = float(np.mean(d * d))
    return float("inf") if mse == 0 else 10.0 * np.log10(peak * peak / mse)


def psnr_yuv(y0, uv0, y1, uv1):
    """(Y, U, V, weighted 6:1:1) PSNR of two NV12 frames."""
    py = psnr(y0, y1)
    pu = psnr(uv0[:, 0::2], uv1[:, 0::2])
    pv = psnr(uv0[:, 1::2], uv1[:, 1::2])
    return py, pu, pv, (6 * py + pu + pv) / 8.0


def bd_rate(rate_anchor, psnr_anchor, rate_test, psnr_test):
    """Bjontegaard delta rate of `test` against `anchor`, in percent."""
    ra, da = np.log(np.asarray(rate_anchor, np.float64)), np.asarray(psnr_anchor, np.float64)
    rt, dt = np.log(np.asarray(rate_test, np.float64)), np.asarray(psnr_test, np.float64)
    if len(ra) < 4 or len(rt) < 4:
        raise ValueError("BD-rate needs four RD points per curve")
    pa = np.polyfit(da, ra, 3)
    pt = np.polyfit(dt, rt, 3)
    lo, hi = max(da.min(), dt.min()), min(da.max(), dt.max())
    if hi <= lo:
        raise ValueError("RD curves do not overlap in PSNR")
    ia, it = np.polyint(pa), np.polyint(pt)
    avg_a = (np.polyval(ia, hi) - np.polyval(ia, lo)) / (hi - lo)
    avg_t = (np.polyval(it, hi) - np.polyval(it, lo)) / (hi - lo)
    return float((np.exp(avg_t - avg_a) - 1.0) * 100.0)
