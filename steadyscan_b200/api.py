"""Python mirror of the reference's ``align_group_to_template`` MEX interface.

``align_group_to_template(flags, template_image, xgrad, ygrad, tfrac, basex, basey, base_mask, bmData,
est_dx_knots, est_dy_knots, group_size, nFrames, min_points_per_block, max_iter, move_thresh,
halt_correlation, correlation_increase_threshold, filter_strength, max_filter_iterations,
filter_deactivation_threshold, lambda, linesearch_reduction_multiplier, solver_id, filter_id,
gpu_device_id, nargout=6)`` takes the 26 arguments of the MEX call (steady_scan.m:239-242,
mex/mexgateway.cpp:38-174) and returns its first ``nargout`` outputs
``(dx_knots, dy_knots, frame_corr, iter_used, mask, residrms, ...)`` (mexgateway.cpp:266-354).
All work runs in the CUDA library through its C ABI; errors raise :class:`SteadyScanError` with
the library's message. ``align_group`` / ``align_groups`` take the argument dict built by
:func:`steadyscan_b200.prep.boundary_arguments` and return dicts; ``align_groups`` runs many groups
in one batched GPU run.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import (SS_DEVICE, SS_F16, SS_F32, SS_F64, SS_HOST, SS_I32, SS_U8, SS_U16, STOP_NAMES, SSInputs,
                   SSMatrix, SSOutputs, SSPrepFrames, SSReconstruct, SteadyScanError, check, load)

__all__ = ["align_group_to_template", "align_group", "align_groups", "estimate_displacements", "recording_sets",
           "prepare_frames", "reconstruct_frames", "DeviceMatrix", "SteadyScanError", "ARG_NAMES", "STOP_NAMES"]

ARG_NAMES = ["flags", "template_image", "xgrad", "ygrad", "tfrac", "basex", "basey", "base_mask", "bmData",
             "est_dx_knots", "est_dy_knots", "group_size", "nFrames", "min_points_per_block", "max_iter",
             "move_thresh", "halt_correlation", "correlation_increase_threshold", "filter_strength",
             "max_filter_iterations", "filter_deactivation_threshold", "lambda", "linesearch_reduction_multiplier",
             "solver_id", "filter_id", "gpu_device_id"]

_NP_DTYPE = {np.dtype(np.float64): SS_F64, np.dtype(np.float32): SS_F32, np.dtype(np.uint16): SS_U16,
             np.dtype(np.float16): SS_F16, np.dtype(np.uint8): SS_U8, np.dtype(np.bool_): SS_U8,
             np.dtype(np.int32): SS_I32}
_TORCH_DTYPE = {"torch.float64": SS_F64, "torch.float32": SS_F32, "torch.uint16": SS_U16,
                "torch.float16": SS_F16, "torch.uint8": SS_U8, "torch.int32": SS_I32}


class DeviceMatrix:
    """A column-major matrix already in device memory: ``ptr`` to ``rows * cols`` elements."""

    def __init__(self, ptr: int, rows: int, cols: int, dtype: int, owner=None):
        self.ptr, self.rows, self.cols, self.dtype, self.owner = int(ptr), int(rows), int(cols), int(dtype), owner


def _matrix(a, keep: list, memo: dict | None = None) -> SSMatrix:
    """ss_matrix of ``a``; with ``memo`` the same Python object maps to the same buffer, so groups
    that share an argument share it in the library too."""
    if memo is not None:
        hit = memo.get(id(a))
        if hit is not None and hit[0] is a:
            return hit[1]
        m = _matrix(a, keep)
        memo[id(a)] = (a, m)
        return m
    if isinstance(a, DeviceMatrix):
        return SSMatrix(a.ptr, a.rows, a.cols, a.dtype, SS_DEVICE)
    if hasattr(a, "is_cuda") and a.is_cuda:  # torch tensor in column-major memory order
        t = a
        if t.dim() == 1:
            rows, cols = t.shape[0], 1
        else:
            rows, cols = t.shape
            if not (t.T.is_contiguous() or cols == 1):
                raise ValueError("device matrices must be column-major (use tensor.T.contiguous().T)")
        keep.append(t)
        return SSMatrix(t.data_ptr(), rows, cols, _TORCH_DTYPE[str(t.dtype)], SS_DEVICE)
    arr = np.asarray(a)
    if arr.dtype not in _NP_DTYPE:
        arr = arr.astype(np.float64)
    if arr.dtype == np.bool_:
        arr = arr.astype(np.uint8)
    if arr.ndim == 0:
        arr = arr.reshape(1, 1)
    elif arr.ndim == 1:
        arr = arr.reshape(-1, 1)
    arr = np.asfortranarray(arr)
    keep.append(arr)
    return SSMatrix(arr.ctypes.data, arr.shape[0], arr.shape[1], _NP_DTYPE[arr.dtype], SS_HOST)


def _inputs(args: dict, template_storage=None, memo: dict | None = None):
    keep: list = []
    flags = args["flags"].encode() if isinstance(args["flags"], str) else bytes(args["flags"])
    keep.append(flags)
    ts = {None: 0, "f32": SS_F32, "f16": SS_F16, np.float32: SS_F32, np.float16: SS_F16}.get(template_storage,
                                                                                          template_storage)
    mp = args["min_points_per_block"]
    i = SSInputs(
        flags,
        _matrix(args["template_image"], keep, memo), _matrix(args["xgrad"], keep, memo),
        _matrix(args["ygrad"], keep, memo), _matrix(args["tfrac"], keep, memo), _matrix(args["basex"], keep, memo),
        _matrix(args["basey"], keep, memo), _matrix(args["base_mask"], keep, memo), _matrix(args["bmData"], keep),
        _matrix(args["est_dx_knots"], keep), _matrix(args["est_dy_knots"], keep), int(args["group_size"]),
        int(args["nFrames"]), _matrix(mp if np.ndim(mp) == 1 else np.asarray(mp).reshape(-1), keep, memo),
        int(args["max_iter"]),
        float(args["move_thresh"]), float(args["halt_correlation"]), float(args["correlation_increase_threshold"]),
        float(args["filter_strength"]), int(args["max_filter_iterations"]),
        float(args["filter_deactivation_threshold"]), float(args.get("lambda", 0.0)),
        float(args["linesearch_reduction_multiplier"]), int(args["solver_id"]), int(args["filter_id"]),
        int(args["gpu_device_id"]), int(ts or 0), int(args.get("frames_per_cta", 0) or 0))
    return i, keep


def _outputs(args: dict, want_mask=True, want_history=False):
    hb, w = np.asarray(args["tfrac"]).shape if not hasattr(args["tfrac"], "shape") else tuple(args["tfrac"].shape)
    nF = int(args["nFrames"])
    N = w * nF + 1
    mi = int(args["max_iter"])
    flags = args["flags"] if isinstance(args["flags"], str) else bytes(args["flags"]).decode()
    letters = flags[1:]  # after the precision letter
    # outputs the library writes in full are left uninitialised; flag p's frame-ordered layout leaves
    # dx/dy unwritten, and the knot layouts of flags P and p exist only with those flags
    knots = np.zeros if "p" in letters else np.empty
    a = dict(dx=knots((w + 1) * nF), dy=knots((w + 1) * nF), frame_corr=np.empty(nF),
             iter_used=np.zeros(1, np.int32), residrms=np.empty(nF), device_init_time=np.zeros(1),
             blocks_used=np.empty(w * nF, np.uint8))
    if "P" in letters:
        a["raw_params"] = np.zeros(2 * N)
    if "p" in letters:
        a["frame_params"] = np.zeros(2 * (w + 1) * nF)
    if want_mask:
        a["mask"] = np.empty(hb * w * nF, np.uint8)
    # outputs 9, 10 and 14 exist with the timing flags (mexgateway.cpp:266-300, task.cpp:242-248)
    if "t" in letters:
        a["rg_params"] = np.empty(2 * N * 2 * mi)
    if "t" in letters or "T" in letters:
        a["function_times"] = np.empty(14)
    if "t" in letters and "T" in letters:
        a["iteration_times"] = np.empty(mi)
    if want_history:
        a["iteration_corr"] = np.zeros(mi)
        a["frame_corr_history"] = np.zeros(nF * mi)
        a["iteration_errvals"] = np.zeros(2 * mi * nF)
        a["all_params"] = np.zeros(2 * N * mi)
    p = lambda k: a[k].ctypes.data if k in a else None
    o = SSOutputs(p("dx"), p("dy"), p("frame_corr"), p("iter_used"), p("mask"), p("residrms"),
                  p("device_init_time"), p("iteration_corr"), p("frame_corr_history"), p("iteration_errvals"),
                  p("raw_params"), p("all_params"), p("frame_params"), 0, 0, 0, 0.0, p("blocks_used"),
                  p("iteration_times"), p("function_times"), p("rg_params"))
    return o, a, (hb, w, nF, N, mi)


def _result(o: SSOutputs, a: dict, dims) -> dict:
    hb, w, nF, N, mi = dims
    r = dict(dx=a["dx"], dy=a["dy"], frame_corr=a["frame_corr"], iter_used=int(a["iter_used"][0]),
             residrms=a["residrms"], device_init_time=float(a["device_init_time"][0]),
             stop_reason=int(o.stop_reason), stop_name=STOP_NAMES[o.stop_reason] if 0 <= o.stop_reason < 5 else "?",
             trial_cap_hit=bool(o.trial_cap_hit), n_frame_passes=int(o.n_frame_passes),
             elapsed_ms=float(o.elapsed_ms), raw_params=a.get("raw_params"),
             frame_params=a["frame_params"].reshape(nF, 2 * (w + 1), order="F") if "frame_params" in a else None,
             blocks_used=a["blocks_used"].reshape(w, nF, order="F").astype(bool))
    if "mask" in a:
        r["mask"] = a["mask"].reshape(hb, w * nF, order="F").astype(bool)
    r["rg_params"] = a["rg_params"].reshape(2 * N, 2 * mi, order="F") if "rg_params" in a else None
    r["function_times"] = a.get("function_times")
    r["iteration_times"] = a.get("iteration_times")
    if "iteration_corr" in a:
        r["iteration_corr"] = a["iteration_corr"]
        r["frame_corr_history"] = a["frame_corr_history"].reshape(nF, mi, order="F")
        r["iteration_errvals"] = a["iteration_errvals"].reshape(2 * mi, nF, order="F")
        r["all_params"] = a["all_params"].reshape(2 * N, mi, order="F")
    return r


def _batch_args(groups, want_mask, want_history, template_storage, memo: dict | None = None):
    n = len(groups)
    ins = (SSInputs * n)()
    outs = (SSOutputs * n)()
    keep, arrays, dims = [], [], []
    memo = {} if memo is None else memo
    for k, g in enumerate(groups):
        i, kk = _inputs(g, template_storage, memo)
        ins[k] = i
        keep.append(kk)
        o, a, d = _outputs(g, want_mask, want_history)
        outs[k] = o
        arrays.append(a)
        dims.append(d)
    return ins, outs, keep, arrays, dims


def align_groups(groups: list, want_mask: bool = True, want_history: bool = False, template_storage=None) -> list:
    """Runs many groups (argument dicts) in one batched run on one GPU; returns a list of dicts."""
    lib = load()
    n = len(groups)
    ins = (SSInputs * n)()
    outs = (SSOutputs * n)()
    keep, arrays, dims = [], [], []
    memo: dict = {}
    for k, g in enumerate(groups):
        i, kk = _inputs(g, template_storage, memo)
        ins[k] = i
        keep.append(kk)
        o, a, d = _outputs(g, want_mask, want_history)
        outs[k] = o
        arrays.append(a)
        dims.append(d)
    check(lib.ss_align_groups(n, ins, outs))
    return [_result(outs[k], arrays[k], dims[k]) for k in range(n)]


def align_group(args: dict, want_mask: bool = True, want_history: bool = False, template_storage=None) -> dict:
    """One align_group_to_template call from the argument dict; returns a dict of outputs."""
    lib = load()
    i, keep = _inputs(args, template_storage)
    o, a, d = _outputs(args, want_mask, want_history)
    check(lib.ss_align_group_to_template(C.byref(i), C.byref(o)))
    del keep
    return _result(o, a, d)


def align_group_to_template(*argv, nargout: int = 6, template_storage=None):
    """MEX-style call with the 26 positional arguments; returns the first ``nargout`` outputs."""
    if len(argv) < 26:
        raise SteadyScanError(-1, f"not enough input arguments, expected 26 - received {len(argv)}")
    args = dict(zip(ARG_NAMES, argv[:26]))
    r = align_group(args, want_mask=nargout >= 5, want_history=nargout >= 8, template_storage=template_storage)
    outs = [r["dx"], r["dy"], r["frame_corr"], np.int32(r["iter_used"]), r.get("mask"), r["residrms"],
            r["device_init_time"]]
    if nargout >= 8:
        outs += [r["iteration_corr"], None, None, r["frame_corr_history"], r["iteration_errvals"], r["raw_params"],
                 None, r["all_params"]]
    return tuple(outs[:nargout])


def prepare_frames(frames, layout, pregauss: float = 0.0, mednorm: bool = False, out_dtype=np.float64,
                   device: int = 0, n_frames: int | None = None):
    """The reference driver's preparation of raw frames on the GPU (ss_prepare_frames):
    prefilter_foralignment (Gaussian blur of std ``pregauss``, then division by each frame's median
    when ``mednorm``; steady_scan.m:625-643), cropimage and image2blockmatrix (steady_scan.m:229-234)
    of every frame. ``frames``: H x W x n (numpy in any memory order, or a CUDA tensor whose frames
    are column-major, i.e. ``t.permute(2, 1, 0)`` contiguous, or a DeviceMatrix of H x (W * n));
    ``layout``: prep.BlockLayout (block map and cropping); ``n_frames`` is needed for a DeviceMatrix.
    Returns the block matrix
    frame_h x (frame_w * n) as a column-major CUDA tensor of ``out_dtype`` (float64, float32, or
    uint16 for uint16 frames without prefilter)."""
    import torch

    from . import prep
    lib = load()
    keep = []
    if isinstance(frames, DeviceMatrix):
        if not n_frames:
            raise ValueError("n_frames is needed for a DeviceMatrix of frames")
        fm = SSMatrix(frames.ptr, frames.rows, frames.cols, frames.dtype, SS_DEVICE)
        n = int(n_frames)
    elif hasattr(frames, "is_cuda") and frames.is_cuda:
        t = frames if frames.dim() == 3 else frames[:, :, None]
        if not t.permute(2, 1, 0).is_contiguous():
            raise ValueError("CUDA frames must be column-major per frame (t.permute(2, 1, 0) contiguous)")
        keep.append(t)
        h, w, n = t.shape
        fm = SSMatrix(t.data_ptr(), h, w * n, _TORCH_DTYPE[str(t.dtype)], SS_DEVICE)
    else:
        a = np.asarray(frames)
        if a.ndim == 2:
            a = a[:, :, None]
        if a.dtype not in _NP_DTYPE or a.dtype in (np.bool_, np.uint8, np.int32):
            a = a.astype(np.float64)
        a = np.asfortranarray(a)
        keep.append(a)
        h, w, n = a.shape
        fm = SSMatrix(a.ctypes.data, h, w * n, _NP_DTYPE[a.dtype], SS_HOST)
    gidx = getattr(layout, "_gather_i32", None)  # the layout's gather map, built once per layout
    if gidx is None:
        gidx = np.asfortranarray(prep._block_gather_index(layout.prevknotind, layout.frame_w).astype(np.int32))
        try:
            layout._gather_i32 = gidx
        except AttributeError:
            pass
    hb, nb = gidx.shape
    tdt = {np.dtype(np.float64): torch.float64, np.dtype(np.float32): torch.float32,
           np.dtype(np.uint16): torch.uint16}[np.dtype(out_dtype)]
    out = torch.empty((nb * n, hb), dtype=tdt, device=f"cuda:{device}").T  # column-major hb x (nb n)
    odt = {torch.float64: SS_F64, torch.float32: SS_F32, torch.uint16: SS_U16}[tdt]
    om = SSMatrix(out.data_ptr(), hb, nb * n, odt, SS_DEVICE)
    crop = layout.cropping if layout.cropping else [0, 0, 0, 0]
    p = SSPrepFrames(fm, int(n), float(pregauss), int(bool(mednorm)), (C.c_int32 * 4)(*[int(c) for c in crop]),
                     gidx.ctypes.data, int(hb), int(nb), om, int(device))
    check(lib.ss_prepare_frames(C.byref(p)))
    del keep
    return out


def reconstruct_frames(frames, dx_knots, dy_knots, settings: dict, template_shape, out_dtype=np.float32,
                       device: int = 0) -> dict:
    """invert_bilinear_sampling of the reference's driver for one set of frames
    (ss_reconstruct_frames, steady_scan.m:290-404): ``frames`` h x w x n (cropped, prefiltered;
    FP32 or FP64 numpy, or a CUDA tensor column-major per frame), ``dx_knots``/``dy_knots`` nknots x
    n, ``settings`` from prep.init_settings (basex, basey, tfrac, prevknotind, ibs_regfac,
    ibs_template_pixel_aspect_ratio), ``template_shape`` (th, tw). Returns the corrected frames
    (th x tw x n numpy of out_dtype, NaN where unconstrained), the mask and the sweeps per frame."""
    lib = load()
    keep = []
    if hasattr(frames, "is_cuda") and frames.is_cuda:
        t = frames if frames.dim() == 3 else frames[:, :, None]
        if not t.permute(2, 1, 0).is_contiguous():
            raise ValueError("CUDA frames must be column-major per frame (t.permute(2, 1, 0) contiguous)")
        keep.append(t)
        h, w, n = t.shape
        fm = SSMatrix(t.data_ptr(), h, w * n, _TORCH_DTYPE[str(t.dtype)], SS_DEVICE)
    else:
        a = np.asarray(frames)
        if a.ndim == 2:
            a = a[:, :, None]
        if a.dtype not in (np.float32, np.float64):
            a = a.astype(np.float32)
        a = np.asfortranarray(a)
        keep.append(a)
        h, w, n = a.shape
        fm = SSMatrix(a.ctypes.data, h, w * n, _NP_DTYPE[a.dtype], SS_HOST)
    th, tw = (int(v) for v in template_shape)
    out = np.empty((th, tw, n), dtype=out_dtype, order="F")
    mask = np.empty((th, tw, n), dtype=np.uint8, order="F")
    iters = np.zeros(n, np.int32)

    def mat(x, dt=np.float64):
        arr = np.asfortranarray(np.asarray(x, dtype=dt))
        if arr.ndim == 1:
            arr = arr.reshape(-1, 1)
        keep.append(arr)
        return SSMatrix(arr.ctypes.data, arr.shape[0], arr.shape[1], _NP_DTYPE[arr.dtype], SS_HOST)

    r = SSReconstruct(fm, int(n), mat(settings["basex"]), mat(settings["basey"]), mat(settings["tfrac"]),
                      mat(settings["prevknotind"], np.int32), mat(dx_knots), mat(dy_knots), th, tw,
                      float(settings.get("ibs_regfac", 3e-3)), float(settings.get("ibs_template_pixel_aspect_ratio", 1.0)),
                      SSMatrix(out.ctypes.data, th, tw * n, _NP_DTYPE[out.dtype], SS_HOST), mask.ctypes.data,
                      iters.ctypes.data, int(device))
    check(lib.ss_reconstruct_frames(C.byref(r)))
    del keep
    return {"data_corrected": out, "mask": mask.astype(bool), "iterations": iters}


def recording_sets(n_frames: int, frames_per_set: int = 500, min_frames_per_set: int = 100):
    """The set split of the reference's driver as its estimate loop uses it (ss_recording_sets):
    a list of (first frame, frame count) per set, 0-based, the overlap frame included."""
    lib = load()
    n = C.c_int32()
    check(lib.ss_recording_sets(int(n_frames), int(frames_per_set), int(min_frames_per_set), None, None, 0,
                                C.byref(n)))
    first = (C.c_int32 * n.value)()
    count = (C.c_int32 * n.value)()
    check(lib.ss_recording_sets(int(n_frames), int(frames_per_set), int(min_frames_per_set), first, count, n.value,
                                C.byref(n)))
    return [(int(first[k]), int(count[k])) for k in range(n.value)]


def estimate_displacements(args: dict, frames_per_set: int = 500, min_frames_per_set: int = 100,
                           corr_thresh: float = 0.75, minblockfrac: float = 0.25, per_set_estimates: bool = False,
                           template_storage=None) -> dict:
    """The reference driver's estimate loop over a whole recording (ss_estimate_displacements,
    steady_scan.m:157-288): ``args`` are the boundary arguments with every frame of the recording in
    ``bmData`` and ``nFrames`` their count. Returns ``dx_knots``/``dy_knots`` (nknots x n_frames),
    ``corr``, ``iter_used``, ``residrms`` (NaN where not estimated: the recording's last frame),
    ``failed``, ``blocks_used`` ((nknots-1) x n_frames) and ``n_sets``."""
    from ._lib import SSRecording, SSRecordingOutputs
    lib = load()
    i, keep = _inputs(args, template_storage)
    rec = SSRecording(i, int(frames_per_set), int(min_frames_per_set), float(corr_thresh), float(minblockfrac),
                      1 if per_set_estimates else 0)
    hb, w = np.shape(args["tfrac"])
    n = int(args["nFrames"])
    a = dict(dx=np.zeros((w + 1) * n), dy=np.zeros((w + 1) * n), corr=np.zeros(n), iter_used=np.zeros(n),
             residrms=np.zeros(n), failed=np.zeros(n, np.uint8), blocks_used=np.zeros(w * n, np.uint8))
    o = SSRecordingOutputs(*[a[k].ctypes.data for k in ("dx", "dy", "corr", "iter_used", "residrms", "failed",
                                                        "blocks_used")], 0)
    check(lib.ss_estimate_displacements(C.byref(rec), C.byref(o)))
    del keep
    return dict(dx_knots=a["dx"].reshape(w + 1, n, order="F"), dy_knots=a["dy"].reshape(w + 1, n, order="F"),
                corr=a["corr"], iter_used=a["iter_used"], residrms=a["residrms"], failed=a["failed"].astype(bool),
                blocks_used=a["blocks_used"].reshape(w, n, order="F").astype(bool), n_sets=int(o.n_sets))


def solve_block_tridiagonal(diag, coupling, rhs, stream: int = 0):
    """FP64 block-tridiagonal solve on the GPU (ss_solve_block_tridiagonal).

    diag (n, 3), coupling (n-1, 4) and rhs (n, 2) are float64 torch CUDA tensors (or arrays, copied
    to the current device); returns x (n, 2) as a torch CUDA tensor."""
    import torch
    d = torch.as_tensor(diag, dtype=torch.float64, device="cuda").contiguous()
    c = torch.as_tensor(coupling, dtype=torch.float64, device="cuda").contiguous()
    b = torch.as_tensor(rhs, dtype=torch.float64, device="cuda").contiguous()
    x = torch.empty_like(b)
    n = d.shape[0]
    lib = load()
    torch.cuda.synchronize()
    check(lib.ss_solve_block_tridiagonal(n, d.data_ptr(), c.data_ptr() if c.numel() else None, b.data_ptr(),
                                         x.data_ptr(), stream or None))
    return x


def solve_block_tridiagonal_noalloc(diag, coupling, rhs, stream: int = 0):
    """The same solve through ss_solve_block_tridiagonal_noalloc, which allocates no device memory:
    its workspace is a fixed array inside the library (at most 32768 blocks). For callers that
    cannot allocate while they run, e.g. a streaming acquisition loop in which cudaMalloc would
    synchronize the device. Calls that overlap on the GPU race on that array."""
    import torch
    d = torch.as_tensor(diag, dtype=torch.float64, device="cuda").contiguous()
    c = torch.as_tensor(coupling, dtype=torch.float64, device="cuda").contiguous()
    b = torch.as_tensor(rhs, dtype=torch.float64, device="cuda").contiguous()
    x = torch.empty_like(b)
    lib = load()
    torch.cuda.synchronize()
    check(lib.ss_solve_block_tridiagonal_noalloc(d.shape[0], d.data_ptr(), c.data_ptr() if c.numel() else None,
                                                 b.data_ptr(), x.data_ptr(), stream or None))
    return x


class Session:
    """One imaging session's template, gradients and scan geometry resident on the device
    (ss_session_*): ``proto`` is an argument dict whose fields 1-7 and 13, precision and device are
    used (frames and knots are ignored)."""

    def __init__(self, proto: dict, template_storage=None):
        self._lib = load()
        i, keep = _inputs(proto, template_storage)
        self._keep = keep
        self.template_storage = template_storage
        h = C.c_void_p()
        check(self._lib.ss_session_create(C.byref(i), C.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ss_session_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _session_array(sessions, n):
    if not sessions:
        return None
    arr = (C.c_void_p * n)()
    for k, s in enumerate(sessions):
        arr[k] = s.handle if s is not None else None
    return arr


class Batch:
    """A prepared batch of groups (ss_batch_*): inputs resident on the device, runnable repeatedly.
    ``sessions`` (one entry per group, or None) use resident session buffers; ``arena`` (device
    pointer, bytes) places the batch in the caller's device memory."""

    def __init__(self, groups: list, want_mask: bool = False, want_history: bool = False, template_storage=None,
                 sessions=None, arena=None):
        from ._lib import SSBatchStats  # noqa: F401
        self._lib = load()
        n = len(groups)
        self._ins, self._outs, self._keep, self._arrays, self._dims = _batch_args(groups, want_mask, want_history,
                                                                                 template_storage)
        self._ses = _session_array(sessions, n)
        h = C.c_void_p()
        if sessions is None and arena is None:
            check(self._lib.ss_batch_create(n, self._ins, self._outs, C.byref(h)))
        else:
            ptr, nbytes = arena if arena is not None else (None, 0)
            check(self._lib.ss_batch_create_ex(n, self._ins, self._outs, self._ses, ptr, nbytes, C.byref(h)))
        self._h = h

    @staticmethod
    def measure(groups: list, want_mask: bool = False, want_history: bool = False, template_storage=None,
                sessions=None, memo: dict | None = None) -> int:
        """Device bytes a Batch of these groups needs (nothing allocated). ``memo`` reuses matrices
        converted by earlier calls for the same argument objects (kept alive by the caller)."""
        lib = load()
        ins, outs, keep, arrays, dims = _batch_args(groups, want_mask, want_history, template_storage, memo)
        nb = C.c_int64()
        check(lib.ss_batch_measure(len(groups), ins, outs, _session_array(sessions, len(groups)), C.byref(nb)))
        return int(nb.value)

    def run(self):
        check(self._lib.ss_batch_run(self._h))

    def start(self):
        check(self._lib.ss_batch_start(self._h))

    def step(self):
        check(self._lib.ss_batch_step(self._h))

    def poll(self) -> int:
        """0 while the launch runs, 1 when the next (host-launched) cycle is due, 2 when every group stopped."""
        rc = self._lib.ss_batch_poll(self._h)
        if rc < 0:
            check(rc)
        return rc

    def collect(self) -> list:
        check(self._lib.ss_batch_collect(self._h))
        return [_result(self._outs[k], self._arrays[k], self._dims[k]) for k in range(len(self._dims))]

    def set_timing(self, on: bool):
        check(self._lib.ss_batch_set_timing(self._h, 1 if on else 0))

    def set_graph(self, on: bool):
        """True (default): the whole run as one CUDA graph; False: one host-launched cycle per step."""
        check(self._lib.ss_batch_set_graph(self._h, 1 if on else 0))

    def stats(self) -> dict:
        from ._lib import SSBatchStats
        st = SSBatchStats()
        check(self._lib.ss_batch_stats_get(self._h, C.byref(st)))
        return dict(n_groups=st.n_groups, cycles=st.cycles, linesearch_rounds=st.linesearch_rounds,
                    kernel_launches=st.kernel_launches, frame_passes=list(st.frame_passes),
                    eval_ms=list(st.eval_ms), arena_bytes=st.arena_bytes, run_ms=st.run_ms,
                    staging=dict(zip(("eval_ctas", "eval_windowed", "ls_ctas", "ls_windowed", "ls_pairs",
                                      "eval_pair_columns"), list(st.staging))),
                    assembly_columns_kept=int(st.assembly_columns_kept))

    @property
    def stream_ptr(self) -> int:
        return int(self._lib.ss_batch_stream(self._h) or 0)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ss_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()
