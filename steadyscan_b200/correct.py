"""Motion-corrected frames from estimated knots, for accuracy reports.

Each frame pixel is placed at the template position its knots give (the warp model of the
alignment: x = basex + dx_c (1 - f) + dx_{c+1} f, task_applyparameters.cuh:33-62) and its value is
splatted bilinearly onto the template grid; the corrected frame is the weighted mean per grid point.
This is a simple stand-in for the reference's resampling (steady_scan.m:290-404), used to compare
knot sets by the frames they produce ("corrected-frame relative L2"), not a port of it.
"""
from __future__ import annotations

import numpy as np


def frame_knots(dx: np.ndarray, dy: np.ndarray, n_frames: int):
    """Per-frame (W+1)-knot vectors from the (W+1)*nF output vectors of the alignment."""
    kx = np.asarray(dx, dtype=np.float64).reshape(n_frames, -1)
    ky = np.asarray(dy, dtype=np.float64).reshape(n_frames, -1)
    return kx, ky


def correct_frames(bm_data, dx, dy, tfrac, basex, basey, base_mask, n_frames: int, template_shape):
    """Corrected frames (nF x Ht x Wt) and their splat weights (same shape) from block-matrix frames
    (Hb x W*nF) and the alignment's dx, dy outputs."""
    ht, wt = template_shape
    tfrac = np.asarray(tfrac, dtype=np.float64)
    bx = np.asarray(basex, dtype=np.float64)
    by = np.asarray(basey, dtype=np.float64)
    bm = np.asarray(base_mask).astype(bool)
    hb, w = tfrac.shape
    data = np.asarray(bm_data)
    kx, ky = frame_knots(dx, dy, n_frames)
    out = np.zeros((n_frames, ht, wt))
    wts = np.zeros((n_frames, ht, wt))
    for f in range(n_frames):
        x = bx + kx[f, :-1][None, :] * (1 - tfrac) + kx[f, 1:][None, :] * tfrac
        y = by + ky[f, :-1][None, :] * (1 - tfrac) + ky[f, 1:][None, :] * tfrac
        v = data[:, f * w:(f + 1) * w].astype(np.float64)
        ok = bm & (x >= 0) & (x < wt - 1) & (y >= 0) & (y < ht - 1)
        x, y, v = x[ok], y[ok], v[ok]
        ix, iy = np.floor(x).astype(np.int64), np.floor(y).astype(np.int64)
        fx, fy = x - ix, y - iy
        num = np.zeros(ht * wt)
        den = np.zeros(ht * wt)
        for ddy, ddx, wgt in ((0, 0, (1 - fx) * (1 - fy)), (0, 1, fx * (1 - fy)), (1, 0, (1 - fx) * fy),
                              (1, 1, fx * fy)):
            idx = (iy + ddy) * wt + (ix + ddx)
            num += np.bincount(idx, weights=wgt * v, minlength=ht * wt)
            den += np.bincount(idx, weights=wgt, minlength=ht * wt)
        with np.errstate(invalid="ignore", divide="ignore"):
            out[f] = np.where(den > 0, num / np.maximum(den, 1e-300), 0.0).reshape(ht, wt)
        wts[f] = den.reshape(ht, wt)
    return out, wts


def relative_l2(corr_a, w_a, corr_b, w_b, min_weight: float = 0.5) -> float:
    """||a - b|| / ||b|| over grid points that both corrections cover with weight >= min_weight."""
    m = (w_a >= min_weight) & (w_b >= min_weight)
    if not m.any():
        return float("nan")
    d = corr_a[m] - corr_b[m]
    return float(np.sqrt(np.sum(d * d) / np.sum(corr_b[m] ** 2)))
