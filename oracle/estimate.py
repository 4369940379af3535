"""CPU restatement of the reference driver's estimate loop: TEST INFRASTRUCTURE ONLY.

Restates ``estimate_displacements`` of steady_scan.m (the set split of steady_scan.m:97-108, the
per-set loop of :216-244 and the post-estimate rules of :246-284, with ``extend_firstandlast`` of
:615-623) on top of the FP64 oracle (``oracle.align_group`` for each set's MEX call). Only tests use
it, as the checker of ``ss_estimate_displacements``.

``blockmatrix2image`` (called at steady_scan.m:265) is not part of the reference snapshot. Its
use there is read as the inverse of ``image2blockmatrix``: block column b of the set's mask holds the
pixels of block b, so ``histc(prevknotind(image), 1:nknots-1) > 0`` is "block column b has a
valid pixel".
"""
from __future__ import annotations

import numpy as np

from . import oracle


def set_starts(n_frames: int, frames_per_set: int, min_frames_per_set: int):
    """``set_start`` and ``set_size`` of steady_scan.m:97-106 (1-based starts, nframes + 1 appended)."""
    set_start = list(range(1, n_frames + 1, frames_per_set))
    set_start.append(n_frames + 1)
    set_size = [b - a for a, b in zip(set_start[:-1], set_start[1:])]
    if len(set_size) > 1 and set_size[-1] < min_frames_per_set:
        mid = (set_size[-2] + set_size[-1]) / 2
        set_size[-2] = int(np.ceil(mid))
        set_size[-1] = int(np.floor(mid))
    return set_start, set_size


def sets(n_frames: int, frames_per_set: int, min_frames_per_set: int):
    """(0-based first frame, frame count) of each set as the estimate loop reads them: set iset covers
    ``set_start(iset):min(set_start(iset + 1), nframes)`` (steady_scan.m:220); the rebalanced
    ``set_size`` only gives the number of sets."""
    set_start, set_size = set_starts(n_frames, frames_per_set, min_frames_per_set)
    out = []
    for iset in range(len(set_size)):
        a = set_start[iset]
        b = min(set_start[iset + 1], n_frames)
        out.append((a - 1, b - a + 1))
    return out


def extend_firstandlast(x, mask):
    """steady_scan.m:615-623."""
    mask = np.asarray(mask, dtype=bool)
    if not mask.any():
        return x
    first = int(np.argmax(mask))
    last = len(mask) - 1 - int(np.argmax(mask[::-1]))
    y = np.array(x, dtype=np.float64)
    y[:first] = x[first]
    y[last + 1:] = x[last]
    return y


def estimate_displacements(args: dict, frames_per_set=500, min_frames_per_set=100, corr_thresh=0.75,
                           minblockfrac=0.25, per_set_estimates=False, n_threads=1) -> dict:
    """The estimate loop over a recording whose frames are all in ``args['bmData']``."""
    hb, w = np.shape(args["tfrac"])
    nk = w + 1
    n = int(args["nFrames"])
    bm = np.asarray(args["bmData"])
    ex_all = np.asarray(args["est_dx_knots"], dtype=np.float64).reshape(nk, -1, order="F")
    ey_all = np.asarray(args["est_dy_knots"], dtype=np.float64).reshape(nk, -1, order="F")
    dx = np.full((nk, n), np.nan)
    dy = np.full((nk, n), np.nan)
    corr = np.full(n, np.nan)
    iters = np.full(n, np.nan)
    resid = np.full(n, np.nan)
    failed = np.zeros(n, dtype=bool)
    used_all = np.zeros((w, n), dtype=bool)
    ss = sets(n, frames_per_set, min_frames_per_set)
    for first, count in ss:
        a = dict(args)
        a["bmData"] = np.asfortranarray(bm[:, first * w:(first + count) * w])
        a["nFrames"] = count
        c0 = first if per_set_estimates else 0  # the MEX reads the first columns (organize2D1)
        a["est_dx_knots"] = ex_all[:, c0:c0 + count]
        a["est_dy_knots"] = ey_all[:, c0:c0 + count]
        o = oracle.align_group(a, n_threads=n_threads)
        for setj in range(count - 1):
            j = first + setj
            dx[:, j] = o["dx"][setj * nk:(setj + 1) * nk]
            dy[:, j] = o["dy"][setj * nk:(setj + 1) * nk]
            corr[j] = o["frame_corr"][setj]
            iters[j] = o["iterations"]
            resid[j] = o["residrms"][setj]
            frame_mask = o["mask"][:, setj * w:(setj + 1) * w]
            used = frame_mask.any(axis=0)
            used_all[:, j] = used
            if not used.any():
                failed[j] = True
                corr[j] = np.nan
                continue
            if not used[0] or not used[-1]:
                dx[:, j] = extend_firstandlast(dx[:, j], used)
                dy[:, j] = extend_firstandlast(dy[:, j], used)
            failed[j] = (not (o["frame_corr"][setj] >= corr_thresh)) or (used.size / (nk - 1) < minblockfrac)
    return dict(dx_knots=dx, dy_knots=dy, corr=corr, iter_used=iters, residrms=resid, failed=failed,
                blocks_used=used_all, n_sets=len(ss))
