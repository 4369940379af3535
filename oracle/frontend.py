"""CPU restatement of the reference driver's frame preparation: TEST INFRASTRUCTURE ONLY.

Restates ``prefilter_foralignment`` (steady_scan.m:625-643) with numpy's FFT the way the reference
writes it (a periodic Gaussian on the frame padded by L rows and columns, multiplied in the
frequency domain, the real part cropped back; then division by each frame's median), ``cropimage``
(steady_scan.m:830-834) and ``image2blockmatrix`` (steady_scan.m:601-613), and the concatenation of
a set's frames into ``bmData`` (steady_scan.m:229-234). Only tests use it, as the checker of
``ss_prepare_frames``.
"""
from __future__ import annotations

import math

import numpy as np


def prefilter_foralignment(data: np.ndarray, gsd: float, mednorm: bool) -> np.ndarray:
    """data: H x W x n; returns FP64 H x W x n (steady_scan.m:625-643)."""
    d = np.array(data, dtype=np.float64, copy=True)
    if d.ndim == 2:
        d = d[:, :, None]
    h, w, n = d.shape
    if gsd > 0:
        L = math.ceil(math.sqrt((2 * gsd ** 2) * math.log(10000 / (math.sqrt(2 * math.pi) * gsd))))
        sb = (h + L, w + L)
        x, y = np.meshgrid(np.arange(1, sb[1] + 1), np.arange(1, sb[0] + 1))
        g2d = np.exp(-(np.minimum(x - 1, sb[1] + 1 - x) ** 2 + np.minimum(y - 1, sb[0] + 1 - y) ** 2) / (2 * gsd ** 2))
        g2d = g2d / g2d.sum()
        G = np.fft.fft2(g2d, s=sb)
        for k in range(n):
            u = np.real(np.fft.ifft2(np.fft.fft2(d[:, :, k], s=sb) * G))
            d[:, :, k] = u[:h, :w]
    if mednorm:
        med = np.median(d.reshape(h * w, n, order="F"), axis=0)
        d = d / med.reshape(1, 1, n)
    return d


def cropimage(x: np.ndarray, cropvec) -> np.ndarray:
    """x(cropvec(3)+1 : end-cropvec(4), cropvec(1)+1 : end-cropvec(2), :) (steady_scan.m:830-834)."""
    l, r, b, t = (int(c) for c in cropvec)
    return x[b:x.shape[0] - t, l:x.shape[1] - r, ...]


def image2blockmatrix(x: np.ndarray, blockind: np.ndarray, nblocks: int):
    """Block matrix of image x: column b holds x(blockind == b) in column-major order, zero padded
    to the largest block (steady_scan.m:601-613); blocks are numbered from 1."""
    xf = np.asarray(x).reshape(-1, order="F")
    bf = np.asarray(blockind).reshape(-1, order="F")
    cols = [xf[bf == b] for b in range(1, nblocks + 1)]
    hb = max(len(c) for c in cols)
    y = np.zeros((hb, nblocks), dtype=xf.dtype)
    for b, c in enumerate(cols):
        y[:len(c), b] = c
    return y


def set_bmdata(frames: np.ndarray, blockind: np.ndarray, nblocks: int, cropping, gsd: float, mednorm: bool):
    """bmData of a set: prefiltered, cropped, block-reordered frames side by side
    (steady_scan.m:229-234)."""
    pre = prefilter_foralignment(frames, gsd, mednorm)
    crop = cropping if cropping is not None and len(cropping) else [0, 0, 0, 0]
    return np.concatenate([image2blockmatrix(cropimage(pre[:, :, k], crop), blockind, nblocks)
                           for k in range(pre.shape[2])], axis=1)
