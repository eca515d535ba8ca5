"""Seeded synthetic video for the encoder's workloads (no dataset is shipped).

Content model, per the workload descriptions the reference is measured on:
smooth gradients, a static Gaussian texture (sigma 8) carried by the
background, six textured rectangles translating at random integer or
quarter-pel velocities of at most 8 px/frame, and optionally a global pan
(0-4 px/frame) plus a high-detail uniform-noise patch covering 10% of the
frame. Frames are 8-bit NV12 (full-resolution Y, interleaved CbCr at half
resolution). Everything derives from numpy's PCG64 seeded from
(seed, stream), so every machine generates identical frames.
"""
import numpy as np


def _bilinear(img, x0, y0, h, w):
    """Samples img at (y0 + i, x0 + j) for an h x w grid, bilinear, edge-clamped."""
    xi = int(np.floor(x0))
    yi = int(np.floor(y0))
    fx, fy = x0 - xi, y0 - yi
    H, W = img.shape
    ys = np.clip(np.arange(yi, yi + h + 1), 0, H - 1)
    xs = np.clip(np.arange(xi, xi + w + 1), 0, W - 1)
    blk = img[np.ix_(ys, xs)]
    top = blk[:-1, :-1] * (1 - fx) + blk[:-1, 1:] * fx
    bot = blk[1:, :-1] * (1 - fx) + blk[1:, 1:] * fx
    return top * (1 - fy) + bot * fy


class Sequence:
    """A deterministic synthetic NV12 sequence of size W x H."""

    def __init__(self, W, H, seed=0, stream=0, pan=False, noise_patch=False, n_rects=6, max_speed=8.0):
        assert W % 2 == 0 and H % 2 == 0
        self.W, self.H = W, H
        rng = np.random.Generator(np.random.PCG64([seed, stream, W, H]))
        self.margin = m = 160 if pan else 16
        ch, cw = H + 2 * m, W + 2 * m
        yy, xx = np.mgrid[0:ch, 0:cw].astype(np.float32)
        g = 128 + 60 * np.sin(xx / (37 + 40 * rng.random()) + 6 * rng.random()) \
            + 40 * np.cos(yy / (53 + 50 * rng.random()) + 6 * rng.random()) \
            + 0.05 * (xx - cw / 2) * rng.uniform(-1, 1)
        g += rng.normal(0.0, 8.0, size=g.shape).astype(np.float32)
        if noise_patch:
            area = 0.10 * W * H
            pw = int(np.sqrt(area * 1.5))
            ph = int(area / pw)
            px = int(rng.integers(m, m + W - pw))
            py = int(rng.integers(m, m + H - ph))
            g[py:py + ph, px:px + pw] = rng.uniform(0, 255, size=(ph, pw))
        self.luma = np.clip(g, 0, 255).astype(np.float32)
        cyy, cxx = np.mgrid[0:ch // 2, 0:cw // 2].astype(np.float32)
        self.cb = np.clip(128 + 40 * np.sin(cxx / 23.0 + rng.random() * 6) + 20 * np.cos(cyy / 31.0), 0, 255).astype(np.float32)
        self.cr = np.clip(128 + 40 * np.cos(cxx / 29.0 + rng.random() * 6) - 20 * np.sin(cyy / 17.0), 0, 255).astype(np.float32)
        self.pan_v = (rng.uniform(0, 4) * np.cos(a := rng.uniform(0, 2 * np.pi)), rng.uniform(0, 4) * np.sin(a)) if pan else (0.0, 0.0)
        self.pan_v = tuple(np.round(np.array(self.pan_v) * 4) / 4)  # quarter-pel
        self.rects = []
        for _ in range(n_rects):
            rw = int(rng.integers(max(8, W // 16), max(9, W // 4)))
            rh = int(rng.integers(max(8, H // 16), max(9, H // 4)))
            tex = np.clip(rng.uniform(40, 215) + 25 * rng.standard_normal((rh + 2, rw + 2)), 0, 255).astype(np.float32)
            vx, vy = rng.uniform(-max_speed, max_speed, size=2)
            if rng.random() < 0.5:
                vx, vy = np.round(vx), np.round(vy)
            else:
                vx, vy = np.round(vx * 4) / 4, np.round(vy * 4) / 4
            self.rects.append(dict(x=float(rng.integers(0, W - rw)), y=float(rng.integers(0, H - rh)), w=rw, h=rh,
                                   vx=float(vx), vy=float(vy), tex=tex, cb=float(rng.uniform(60, 196)),
                                   cr=float(rng.uniform(60, 196))))

    def frame(self, t):
        """Returns (y [H, W], uv [H/2, W]) uint8 arrays of frame t (NV12)."""
        W, H, m = self.W, self.H, self.margin
        ox, oy = m + self.pan_v[0] * t, m + self.pan_v[1] * t
        # keep the pan inside the margin by reflecting its direction
        span = 2 * m - 4
        ox = m + (((ox - m) + span) % (2 * span)) - span if abs(ox - m) > span else ox
        oy = m + (((oy - m) + span) % (2 * span)) - span if abs(oy - m) > span else oy
        y = _bilinear(self.luma, ox, oy, H, W)
        cb = _bilinear(self.cb, ox / 2, oy / 2, H // 2, W // 2)
        cr = _bilinear(self.cr, ox / 2, oy / 2, H // 2, W // 2)
        for r in self.rects:
            x = (r["x"] + r["vx"] * t) % (W + r["w"]) - r["w"]
            yq = (r["y"] + r["vy"] * t) % (H + r["h"]) - r["h"]
            x0, y0 = int(np.floor(x)), int(np.floor(yq))
            fx, fy = x - x0, yq - y0
            tex = _bilinear(r["tex"], 1 - fx, 1 - fy, r["h"], r["w"])
            xa, xb = max(0, x0), min(W, x0 + r["w"])
            ya, yb = max(0, y0), min(H, y0 + r["h"])
            if xa < xb and ya < yb:
                y[ya:yb, xa:xb] = tex[ya - y0:yb - y0, xa - x0:xb - x0]
                cb[ya // 2:(yb + 1) // 2, xa // 2:(xb + 1) // 2] = r["cb"]
                cr[ya // 2:(yb + 1) // 2, xa // 2:(xb + 1) // 2] = r["cr"]
        y8 = np.clip(np.rint(y), 0, 255).astype(np.uint8)
        uv = np.empty((H // 2, W), np.uint8)
        uv[:, 0::2] = np.clip(np.rint(cb), 0, 255).astype(np.uint8)
        uv[:, 1::2] = np.clip(np.rint(cr), 0, 255).astype(np.uint8)
        return y8, uv


def workload(name, seed=0, stream=0):
    """The synthetic generator for a named workload configuration."""
    if name == "h264_640x480":  # plain H.264 Baseline, 640x480
        return Sequence(640, 480, seed, stream)
    if name == "h264_1080p":  # plain H.264 High, 1920x1080, pan + noise patch
        return Sequence(1920, 1080, seed, stream, pan=True, noise_patch=True)
    raise KeyError(name)
