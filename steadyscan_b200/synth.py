"""Seeded synthetic recordings with known ground truth.

The reference ships no data. These generators produce raster-scanned frames of a template under
a known per-line displacement, with the shapes, knot spacings and noise levels of the five
workloads this package is measured on:

* template: Gaussian blobs (amplitude U[0.3, 1], sigma U[s0, s1] px, centres uniform) on a 0.1
  background, scaled so that its peak equals ``peak_photons`` (the expected photon count), so
  template and frames are in the same units;
* displacement: per scan line, a random walk (step N(0, walk_sigma) px per line) in x and y,
  continuous across frames, with jumps of up to ``jump_px`` at uniformly drawn lines, clipped to
  +-``clip_px``;
* frame pixel (line l, column j) = bilinear sample of the template at (j + dx_l, l + dy_l)
  (background outside), then Poisson noise; stored as uint16 / float16 / float32 / float64.

Seeds: the workload with number ``c`` uses ``seed = 1000 + c``.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

__all__ = ["make_template", "make_walk", "render_frames", "Recording", "make_recording",
           "truth_knots", "WORKLOADS"]


def make_template(h: int, w: int, n_blobs: int, sigma=(2.0, 5.0), rng=None,
                  background: float = 0.1, peak_photons: float = 200.0) -> np.ndarray:
    rng = np.random.default_rng(rng)
    yy, xx = np.mgrid[0:h, 0:w].astype(np.float64)
    img = np.full((h, w), background, dtype=np.float64)
    cy = rng.uniform(0, h, n_blobs)
    cx = rng.uniform(0, w, n_blobs)
    sg = rng.uniform(sigma[0], sigma[1], n_blobs)
    amp = rng.uniform(0.3, 1.0, n_blobs)
    for i in range(n_blobs):
        r = int(np.ceil(6 * sg[i]))
        y0, y1 = max(0, int(cy[i]) - r), min(h, int(cy[i]) + r + 1)
        x0, x1 = max(0, int(cx[i]) - r), min(w, int(cx[i]) + r + 1)
        if y0 >= y1 or x0 >= x1:
            continue
        d2 = (yy[y0:y1, x0:x1] - cy[i]) ** 2 + (xx[y0:y1, x0:x1] - cx[i]) ** 2
        img[y0:y1, x0:x1] += amp[i] * np.exp(-d2 / (2 * sg[i] ** 2))
    return img * (peak_photons / img.max())


def make_walk(n_lines_total: int, walk_sigma: float, clip_px: float, jumps_per_frame,
              lines_per_frame: int, jump_px: float, rng=None) -> np.ndarray:
    """Per-line (dx, dy), shape (n_lines_total, 2), continuous across frames."""
    rng = np.random.default_rng(rng)
    steps = rng.normal(0.0, walk_sigma, size=(n_lines_total, 2))
    n_frames = n_lines_total // lines_per_frame
    for f in range(n_frames):
        if isinstance(jumps_per_frame, tuple):
            nj = int(rng.integers(jumps_per_frame[0], jumps_per_frame[1] + 1))
        else:
            nj = int(jumps_per_frame)
        for _ in range(nj):
            line = f * lines_per_frame + int(rng.integers(0, lines_per_frame))
            ang = rng.uniform(0, 2 * np.pi)
            mag = rng.uniform(0, jump_px)
            steps[line] += mag * np.array([np.cos(ang), np.sin(ang)])
    walk = np.empty_like(steps)
    cur = np.zeros(2)
    for i in range(n_lines_total):
        cur = np.clip(cur + steps[i], -clip_px, clip_px)
        walk[i] = cur
    return walk


def _bilinear(template: np.ndarray, x: np.ndarray, y: np.ndarray, background: float) -> np.ndarray:
    h, w = template.shape
    x0 = np.floor(x).astype(np.int64)
    y0 = np.floor(y).astype(np.int64)
    fx = x - x0
    fy = y - y0
    inside = (x0 >= 0) & (y0 >= 0) & (x0 < w - 1) & (y0 < h - 1)
    x0c = np.clip(x0, 0, w - 2)
    y0c = np.clip(y0, 0, h - 2)
    t00 = template[y0c, x0c]
    t01 = template[y0c, x0c + 1]
    t10 = template[y0c + 1, x0c]
    t11 = template[y0c + 1, x0c + 1]
    v = (1 - fx) * ((1 - fy) * t00 + fy * t10) + fx * ((1 - fy) * t01 + fy * t11)
    return np.where(inside, v, background)


def render_frames(template: np.ndarray, walk: np.ndarray, nlines: int, linewidth: int,
                  rng=None, noise: bool = True, background: float | None = None) -> np.ndarray:
    """Frames (nlines x linewidth x n) sampled along ``walk`` (one row per scan line)."""
    rng = np.random.default_rng(rng)
    n = walk.shape[0] // nlines
    bg = float(template.min()) if background is None else background
    out = np.empty((nlines, linewidth, n), dtype=np.float64)
    jj = np.arange(linewidth, dtype=np.float64)[None, :]
    ll = np.arange(nlines, dtype=np.float64)[:, None]
    for f in range(n):
        wl = walk[f * nlines:(f + 1) * nlines]
        x = jj + wl[:, 0:1]
        y = ll + wl[:, 1:2]
        lam = _bilinear(template, x, y, bg)
        out[:, :, f] = rng.poisson(lam) if noise else lam
    return out


def truth_knots(walk: np.ndarray, nlines: int, nknots: int, n_frames: int):
    """Ground truth at knot times: knot k of frame f sits at line f*nlines + k*lpk (the last knot
    of a frame is the first line of the next frame). Returns (dx, dy), each nknots x n_frames."""
    lpk = nlines / (nknots - 1)
    dx = np.empty((nknots, n_frames))
    dy = np.empty((nknots, n_frames))
    total = walk.shape[0]
    for f in range(n_frames):
        for k in range(nknots):
            line = min(int(round(f * nlines + k * lpk)), total - 1)
            dx[k, f] = walk[line, 0]
            dy[k, f] = walk[line, 1]
    return dx, dy


@dataclass
class Recording:
    template: np.ndarray
    frames: np.ndarray            # nlines x linewidth x n (float64 photon counts)
    walk: np.ndarray              # per-line (dx, dy)
    nknots: int
    params: dict = field(default_factory=dict)

    def frames_as(self, dtype) -> np.ndarray:
        if np.dtype(dtype) == np.uint16:
            return np.clip(np.rint(self.frames), 0, 65535).astype(np.uint16)
        return self.frames.astype(dtype)


def make_recording(h: int, w: int, n_frames: int, nknots: int, n_blobs: int, sigma, walk_sigma,
                   clip_px, jumps_per_frame, jump_px: float = 4.0, seed: int = 0,
                   nlines: int | None = None, linewidth: int | None = None,
                   noise: bool = True) -> Recording:
    """Template of ``h x w`` and ``n_frames`` frames of ``nlines x linewidth`` (default h x w)."""
    rng = np.random.default_rng(seed)
    nl = h if nlines is None else nlines
    lw = w if linewidth is None else linewidth
    tmpl = make_template(h, w, n_blobs, sigma, rng)
    walk = make_walk(nl * (n_frames + 1), walk_sigma, clip_px, jumps_per_frame, nl, jump_px, rng)
    frames = render_frames(tmpl, walk[:nl * n_frames], nl, lw, rng, noise=noise)
    return Recording(tmpl, frames, walk, nknots,
                     dict(h=h, w=w, n_frames=n_frames, seed=seed, nlines=nl, linewidth=lw))


# Workload shapes (sizes, knot spacing, noise and motion statistics).
WORKLOADS = {
    1: dict(h=256, w=256, n_frames=50, nknots=65, n_blobs=80, sigma=(2.0, 5.0), walk_sigma=0.15,
            clip_px=6.0, jumps_per_frame=1, jump_px=4.0, lam=1e-2, max_iter=30, seed=1001),
    2: dict(h=512, w=512, n_frames=2000, nknots=257, n_blobs=400, sigma=(2.0, 6.0),
            walk_sigma=0.1, clip_px=10.0, jumps_per_frame=(0, 3), jump_px=4.0, lam=5e-3,
            batch=64, seed=1002),
    3: dict(n_groups=96, sizes=[(128, 128), (256, 512), (512, 512), (796, 512)],
            lines_per_knot=[1, 2, 4], group_len=(1, 128), walk_sigma=0.15, clip_px=6.0,
            jumps_per_frame=1, jump_px=4.0, tol=1e-3, seed=1003),
    4: dict(h=512, w=512, n_frames=4000, nknots=257, n_blobs=400, sigma=(2.0, 6.0),
            walk_sigma=0.15, clip_px=6.0, jumps_per_frame=1, jump_px=4.0, seed=1004),
    5: dict(n_sessions=8, h=512, w=512, group_len=(1, 64), rate_hz=30.0, burst_every_s=10.0,
            burst_factor=2.0, duration_s=60.0, seed=1005),
}
