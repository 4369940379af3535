"""Caller-side preparation of the ``align_group_to_template`` inputs.

These functions restate the host-side set-up that the MATLAB driver performs before it calls the
estimator, so that tests, benchmarks and users can build the 26 boundary arguments from raw frames:

* ``default_alignment_settings``  -- steady_scan.m:836-884
* ``init_settings``               -- steady_scan.m:748-828 (timing model, knot times, tfrac, basex/y)
* ``image2blockmatrix``           -- steady_scan.m:601-613
* ``cropimage``                   -- steady_scan.m:830-834
* ``template_gradients``          -- steady_scan.m:177-179
* ``min_points_per_block``        -- steady_scan.m:174-175
* ``boundary_arguments``          -- steady_scan.m:165-242 (the per-set argument list)

All matrices follow MATLAB conventions: a 2-D numpy array indexed ``[row, col]``; where a flat
order matters it is column-major (Fortran) order, as MATLAB stores it.
"""
from __future__ import annotations

import copy
from dataclasses import dataclass

import numpy as np

__all__ = [
    "default_alignment_settings",
    "init_settings",
    "image2blockmatrix",
    "blockmatrix2image",
    "cropimage",
    "template_gradients",
    "min_points_per_block",
    "matlab_linspace",
    "BlockLayout",
    "block_layout",
    "frames_to_blockmatrix",
    "boundary_arguments",
]


def default_alignment_settings() -> dict:
    """Default settings struct (steady_scan.m:836-867), field for field."""
    return {
        "move_thresh": 0.010,
        "corr_thresh": 0.75,
        "max_iter": 120,
        "nknots": 33,
        "pregauss": 0,
        "mednorm": 0,
        "min_blockpoints_ratio": 0.3,
        "minblockfrac": 0.25,
        "haltcorr": 0.995,
        "isbidirectional": False,
        "linesearch_reduction_multiplier": 0.5,
        "frames_per_set": 500,
        "min_frames_per_set": 100,
        "cropping": [],
        "subrec": [],
        "ibs_inpaint": False,
        "ibs_regfac": 3e-3,
        "ibs_template_pixel_aspect_ratio": 1,
        "ibs_version": 2,
        "gpu_device_id": 0,
        "gpu_frame_groupsize": 2,
        "gpu_correlation_increase_thresh": -1,
        "gpu_solver_id": 2,
        "gpu_filter_id": 1,
        "gpu_filter_strength": 0.8,
        "gpu_filter_max_iterations": 10,
        "gpu_filter_correlation_thresh": 0.01,
        "gpu_forced_precision": "D",
        "gpu_flags": "",
        # Extension of this implementation (the reference hard-codes lambda = 0,
        # steady_scan.m:207-208): weight of the knot-difference regulariser.
        "lambda": 0.0,
    }


def matlab_linspace(d1: float, d2: float, n: int) -> np.ndarray:
    """MATLAB ``linspace`` for finite endpoints: ``d1 + (0:n-1).*(d2-d1)./(n-1)``, ends exact."""
    n = int(n)
    if n < 1:
        return np.zeros(0)
    if n == 1:
        return np.array([float(d2)])
    n1 = n - 1
    i = np.arange(n, dtype=np.float64)
    y = d1 + (i * (d2 - d1)) / n1
    y[0] = d1
    y[-1] = d2
    return y


def cropimage(x: np.ndarray, cropvec) -> np.ndarray:
    """``cropimage`` (steady_scan.m:830-834); ``cropvec`` is [left right bottom top]."""
    c = [int(v) for v in cropvec]
    r0, r1 = c[2], x.shape[0] - c[3]
    c0, c1 = c[0], x.shape[1] - c[1]
    return x[r0:r1, c0:c1, ...]


def _histc_bins(values: np.ndarray, edges: np.ndarray) -> np.ndarray:
    """MATLAB ``[~, bin] = histc(values, edges)``: 1-based bin, ``edges(k) <= v < edges(k+1)``;
    ``v == edges(end)`` goes to the last bin; values outside get 0."""
    v = np.asarray(values, dtype=np.float64)
    idx = np.searchsorted(edges, v, side="right")  # number of edges <= v
    out = idx.astype(np.int64)
    out[v < edges[0]] = 0
    out[v > edges[-1]] = 0
    out[v == edges[-1]] = len(edges)
    return out


def init_settings(settings: dict | None, template: np.ndarray, nlines: int, linewidth: int) -> dict:
    """Timing model and default scan geometry (steady_scan.m:748-828).

    Adds ``prevknotind`` (1-based knot index per pixel), ``tfrac`` (fraction of the way from the
    previous knot to the next, in scan time), ``basex``/``basey`` (1-based template coordinates of
    each undisplaced pixel), plus ``cropping``/``subrec`` defaults.
    """
    defaults = default_alignment_settings()
    if not settings:
        s = copy.deepcopy(defaults)
    else:
        s = dict(settings)
        for k, v in defaults.items():
            if k not in s:
                s[k] = copy.deepcopy(v)

    if s["cropping"] is None or len(s["cropping"]) == 0:
        s["cropping"] = [0, 0, 0, 0]
    else:
        c = np.asarray(s["cropping"], dtype=np.float64)
        if not (np.all(c >= 0) and np.all(np.round(c) == c)):
            raise ValueError("cropping must be defined with positive integers")
    crop = [int(v) for v in s["cropping"]]

    cropped = (nlines - (crop[2] + crop[3]), linewidth - (crop[0] + crop[1]))
    if not (cropped[0] > 0 and cropped[1] > 0):
        raise ValueError("no image pixels left")

    th, tw = template.shape[0], template.shape[1]
    if s["subrec"] is None or len(s["subrec"]) == 0:
        if cropped == (th, tw):
            s["subrec"] = [1 - crop[0], tw + crop[1], 1 - crop[2], th + crop[3]]
        else:
            s["subrec"] = [1, tw, 1, th]
    else:
        sr = s["subrec"]
        if not (sr[0] < sr[1] and sr[2] < sr[3]):
            raise ValueError("subrec is incorrectly described; use [left right bottom top]")

    npixels = nlines * linewidth
    dwell = 1.0 / npixels
    lin = np.arange(npixels, dtype=np.float64).reshape(nlines, linewidth)  # (l, j) -> l*lw + j
    pst = dwell / 2 + lin / npixels
    if s["isbidirectional"]:
        pst[1::2, :] = pst[1::2, ::-1]
    pst_c = cropimage(pst, crop)

    nl = pst_c.shape[0]
    nknots = int(s["nknots"])
    lpk = nl / (nknots - 1)
    if lpk == round(lpk):
        lpk_i = int(round(lpk))
        knotlines = np.arange(0, nl, lpk_i)  # 1:lpk:nlines, 0-based; indexes the uncropped times
        t_knots = np.concatenate([pst[knotlines, :].min(axis=1) - dwell / 2, [1.0]])
        t_knots[0] = 0.0
    else:
        t_knots = matlab_linspace(pst_c.min() - dwell / 2, pst_c.max() + dwell / 2, nknots)
        t_knots[0] = 0.0
        t_knots[-1] = 1.0

    prevknotind = _histc_bins(pst_c, t_knots)
    if not (np.all(prevknotind > 0) and np.all(prevknotind < nknots)):
        raise ValueError(
            "error in setting up interpolation timing, pixel time is out of range with respect to "
            "interpolation knots")
    s["prevknotind"] = prevknotind
    tk = t_knots
    s["tfrac"] = (pst_c - tk[prevknotind - 1]) / (tk[prevknotind] - tk[prevknotind - 1])
    s["t_knots"] = t_knots

    if s.get("basex") is None or s.get("basey") is None or len(np.atleast_1d(s.get("basex"))) == 0 \
            or len(np.atleast_1d(s.get("basey"))) == 0:
        sr = s["subrec"]
        xs = matlab_linspace(0, 1, linewidth) * (sr[1] - sr[0]) + sr[0]
        ys = matlab_linspace(0, 1, nl) * (sr[3] - sr[2]) + sr[2]
        bx, by = np.meshgrid(xs, ys)
        s["basex"] = cropimage(bx, crop)
        s["basey"] = cropimage(by, crop)
        if s["basex"].shape != pst_c.shape:
            # steady_scan.m:820-824 meshes the cropped line count with the uncropped width and then
            # crops again, so with vertical cropping the default geometry does not match the data.
            raise ValueError("default basex/basey do not match the cropped data (vertical cropping); "
                             "pass basex and basey explicitly")
    else:
        bx = np.asarray(s["basex"])
        by = np.asarray(s["basey"])
        if not (bx.shape == cropped or by.shape == cropped):
            raise ValueError("when basex and basey are given as inputs, they must match the size of "
                             "the data after cropping")
    return s


def _block_gather_index(blockind: np.ndarray, nblocks: int):
    """Flat column-major pixel index of entry (row, block) of the block matrix, -1 where empty."""
    bi = np.asarray(blockind).reshape(-1, order="F")
    order = np.argsort(bi, kind="stable")          # column-major order within each block
    counts = np.bincount(bi, minlength=nblocks + 1)
    starts = np.concatenate([[0], np.cumsum(counts)])
    hb = int(counts[1:nblocks + 1].max()) if nblocks > 0 else 0
    idx = np.full((hb, nblocks), -1, dtype=np.int64)
    for b in range(1, nblocks + 1):
        n = int(counts[b])
        idx[:n, b - 1] = order[starts[b]:starts[b] + n]
    return idx


def image2blockmatrix(x: np.ndarray, blockind: np.ndarray, nblocks: int | None = None):
    """One column per block of pixels (steady_scan.m:601-613).

    Pixels of block ``b`` (1-based ``blockind == b``) fill column ``b-1`` in MATLAB column-major
    order of ``x``; ``bmmask`` marks the filled entries. Returns ``(y, bmmask)``.
    """
    xf = np.asarray(x).reshape(-1, order="F")
    if nblocks is None:
        nblocks = int(np.asarray(blockind).max())
    idx = _block_gather_index(blockind, nblocks)
    m = idx >= 0
    y = np.zeros(idx.shape, dtype=xf.dtype)
    y[m] = xf[idx[m]]
    return y, m


def blockmatrix2image(y: np.ndarray, blockind: np.ndarray, bmmask: np.ndarray, shape) -> np.ndarray:
    """Inverse of :func:`image2blockmatrix` for one frame (column-major image order)."""
    bi = np.asarray(blockind).reshape(-1, order="F")
    out = np.zeros(int(np.prod(shape)), dtype=y.dtype)
    nblocks = y.shape[1]
    for b in range(1, nblocks + 1):
        n = int(bmmask[:, b - 1].sum())
        out[bi == b] = y[:n, b - 1]
    return out.reshape(shape, order="F")


def template_gradients(template: np.ndarray):
    """Forward-difference gradients with a NaN last column/row (steady_scan.m:177-179)."""
    t = np.asarray(template, dtype=np.float64)
    xg = np.concatenate([np.diff(t, axis=1), np.full((t.shape[0], 1), np.nan)], axis=1)
    yg = np.concatenate([np.diff(t, axis=0), np.full((1, t.shape[1]), np.nan)], axis=0)
    return np.asfortranarray(xg), np.asfortranarray(yg)  # column-major, as the C ABI reads them


def min_points_per_block(prevknotind: np.ndarray, nknots: int, ratio: float) -> np.ndarray:
    """``histc(prevknotind, 1:nknots) * ratio`` (steady_scan.m:174-175), cast to int32 by
    truncation as the MEX gateway's ``static_cast<int>`` does (mexconverter.cpp:52)."""
    bi = np.asarray(prevknotind).reshape(-1, order="F")
    counts = np.bincount(bi, minlength=nknots + 1)[1:nknots + 1].astype(np.float64)
    return np.trunc(counts * ratio).astype(np.int32)


@dataclass
class BlockLayout:
    """Block-matrix geometry derived from the settings (one frame)."""
    nknots: int
    frame_w: int          # knot blocks per frame (nknots - 1)
    frame_h: int          # max pixels per block
    prevknotind: np.ndarray
    tfrac: np.ndarray     # frame_h x frame_w
    basex: np.ndarray     # 0-based template x, frame_h x frame_w
    basey: np.ndarray     # 0-based template y
    base_mask: np.ndarray
    min_points: np.ndarray  # int32, nknots
    cropping: list


def block_layout(settings: dict) -> BlockLayout:
    """Block matrices of ``tfrac``, ``basex-1``, ``basey-1`` (steady_scan.m:166-175)."""
    nk = int(settings["nknots"])
    pk = settings["prevknotind"]
    tfrac, bmask = image2blockmatrix(settings["tfrac"], pk, nk - 1)
    bx, _ = image2blockmatrix(np.asarray(settings["basex"], dtype=np.float64) - 1, pk, nk - 1)
    by, _ = image2blockmatrix(np.asarray(settings["basey"], dtype=np.float64) - 1, pk, nk - 1)
    mp = min_points_per_block(pk, nk, float(settings["min_blockpoints_ratio"]))
    f = np.asfortranarray  # column-major, as the C ABI reads them (no conversion per call)
    return BlockLayout(nk, nk - 1, tfrac.shape[0], pk, f(tfrac), f(bx), f(by), f(bmask), mp,
                       list(settings["cropping"]))


def frames_to_blockmatrix(frames: np.ndarray, layout: BlockLayout, dtype=None) -> np.ndarray:
    """Concatenate frames (H x W x n) into ``bmData`` = frame_h x (frame_w * n)
    (steady_scan.m:229-234), optionally keeping a storage dtype such as uint16."""
    frames = np.asarray(frames)
    if frames.ndim == 2:
        frames = frames[:, :, None]
    n = frames.shape[2]
    dt = dtype if dtype is not None else np.float64
    out = np.zeros((layout.frame_h, layout.frame_w * n), dtype=dt)
    flat_idx = _block_gather_index(layout.prevknotind, layout.frame_w)
    valid = flat_idx >= 0
    for k in range(n):
        fr = cropimage(frames[:, :, k], layout.cropping).reshape(-1, order="F")
        blk = np.zeros((layout.frame_h, layout.frame_w), dtype=dt)
        blk[valid] = fr[flat_idx[valid]]
        out[:, k * layout.frame_w:(k + 1) * layout.frame_w] = blk
    return out


def boundary_arguments(settings: dict, template: np.ndarray, bm_data: np.ndarray, n_frames: int,
                       est_dx_knots=None, est_dy_knots=None, layout: BlockLayout | None = None,
                       gradients=None):
    """The 26 ``align_group_to_template`` arguments in MEX order (steady_scan.m:195-242), as a dict
    keyed by the reference's variable names. ``gradients`` = (xgrad, ygrad) of ``template`` reuses
    arrays already made, so the groups of one recording pass the same template objects and the
    library uploads them once."""
    lay = layout or block_layout(settings)
    xg, yg = gradients if gradients is not None else template_gradients(template)
    nk = lay.nknots
    if est_dx_knots is None or est_dy_knots is None:
        est_dx_knots = np.zeros((nk, n_frames))
        est_dy_knots = np.zeros((nk, n_frames))
    flags = str(settings["gpu_forced_precision"]) + str(settings["gpu_flags"])
    return {
        "flags": flags,
        "template_image": np.asarray(template, dtype=np.float64),
        "xgrad": xg,
        "ygrad": yg,
        "tfrac": lay.tfrac,
        "basex": lay.basex,
        "basey": lay.basey,
        "base_mask": lay.base_mask,
        "bmData": bm_data,
        # column-major like every matrix of the C ABI (no conversion per call)
        "est_dx_knots": np.asfortranarray(est_dx_knots, dtype=np.float64),
        "est_dy_knots": np.asfortranarray(est_dy_knots, dtype=np.float64),
        "group_size": lay.frame_w * int(settings["gpu_frame_groupsize"]),
        "nFrames": int(n_frames),
        "min_points_per_block": lay.min_points,
        "max_iter": int(settings["max_iter"]),
        "move_thresh": float(settings["move_thresh"]),
        "halt_correlation": float(settings["haltcorr"]),
        "correlation_increase_threshold": float(settings["gpu_correlation_increase_thresh"]),
        "filter_strength": float(settings["gpu_filter_strength"]),
        "max_filter_iterations": int(settings["gpu_filter_max_iterations"]),
        "filter_deactivation_threshold": float(settings["gpu_filter_correlation_thresh"]),
        "lambda": float(settings.get("lambda", 0.0)),
        "linesearch_reduction_multiplier": float(settings["linesearch_reduction_multiplier"]),
        "solver_id": int(settings["gpu_solver_id"]),
        "filter_id": int(settings["gpu_filter_id"]),
        "gpu_device_id": int(settings["gpu_device_id"]),
    }
