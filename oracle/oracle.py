"""Python front of the FP64 CPU oracle (ss_oracle.c): TEST INFRASTRUCTURE ONLY.

Only tests, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg use this module, as the
checker of the CUDA path. It takes the same 26 boundary arguments (MATLAB layout, as built by
``steadyscan_b200.prep.boundary_arguments``) and returns the reference's outputs 1-6.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libss_oracle.so")
_lib = None

STOP_NAMES = ["CorrelationIncreaseThreshold", "HaltCorrelation", "MovementThreshold", "IterationLimit",
              "Error"]


class _In(C.Structure):
    _fields_ = [
        ("flags", C.c_char_p),
        ("templ_h", C.c_int), ("templ_w", C.c_int),
        ("templ", C.c_void_p), ("xgrad", C.c_void_p), ("ygrad", C.c_void_p),
        ("frame_h", C.c_int), ("frame_w", C.c_int), ("n_frames", C.c_int),
        ("frac", C.c_void_p), ("basex", C.c_void_p), ("basey", C.c_void_p),
        ("base_mask", C.c_void_p), ("image", C.c_void_p),
        ("est_dx", C.c_void_p), ("est_dy", C.c_void_p), ("min_points", C.c_void_p),
        ("group_size", C.c_int), ("max_iter", C.c_int),
        ("move_thresh", C.c_double), ("halt_corr", C.c_double), ("corr_inc_thresh", C.c_double),
        ("filter_strength", C.c_double), ("max_filter_iter", C.c_int),
        ("filter_corr_thresh", C.c_double), ("lam", C.c_double), ("ls_mult", C.c_double),
        ("solver_id", C.c_int), ("filter_id", C.c_int), ("n_threads", C.c_int),
    ]


class _Out(C.Structure):
    _fields_ = [
        ("p_last", C.c_void_p), ("dx_knots", C.c_void_p), ("dy_knots", C.c_void_p),
        ("frame_corr", C.c_void_p), ("residrms", C.c_void_p), ("mask", C.c_void_p),
        ("iter_corr", C.c_void_p), ("frame_corr_hist", C.c_void_p), ("iter_errvals", C.c_void_p),
        ("all_params", C.c_void_p), ("n_eval", C.c_void_p),
        ("iterations", C.c_int), ("stop_reason", C.c_int), ("ls_trial_cap_hit", C.c_int),
        ("rg_params", C.c_void_p),
    ]


def build(force: bool = False) -> str:
    """Compile ss_oracle.c with gcc (OpenMP) into oracle/libss_oracle.so."""
    src = os.path.join(_HERE, "ss_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < max(
            os.path.getmtime(src), os.path.getmtime(os.path.join(_HERE, "ss_oracle.h"))):
        subprocess.check_call(["gcc", "-O2", "-fopenmp", "-shared", "-fPIC", "-o", _LIB_PATH, src, "-lm"])
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _lib.sso_align_group.argtypes = [C.POINTER(_In), C.POINTER(_Out)]
        _lib.sso_align_group.restype = C.c_int
        for name in ("sso_smearing_filter", "sso_range_filter"):
            getattr(_lib, name).argtypes = [C.c_void_p, C.c_int, C.c_double]
        _lib.sso_organize2d1.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        _lib.sso_organize1d2.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        _lib.sso_block_tridiag_solve.argtypes = [C.c_int] + [C.c_void_p] * 4
    return _lib


def _rm(a, dtype=np.float64):
    """Row-major contiguous copy (the reference's internal NeutralMatrix RowMajor layout)."""
    return np.ascontiguousarray(np.asarray(a, dtype=dtype))


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


def align_group(args: dict, n_threads: int = 1, want_mask: bool = True, want_history: bool = False):
    """Runs the oracle on the 26 boundary arguments; returns a dict of outputs."""
    L = lib()
    t = _rm(args["template_image"])
    xg = _rm(args["xgrad"])
    yg = _rm(args["ygrad"])
    frac = _rm(args["tfrac"])
    bx = _rm(args["basex"])
    by = _rm(args["basey"])
    bm = _rm(args["base_mask"], np.uint8)
    img = _rm(args["bmData"])
    nF = int(args["nFrames"])
    hb, w = frac.shape
    edx = np.asarray(args["est_dx_knots"], dtype=np.float64).reshape(-1, order="F").copy()
    edy = np.asarray(args["est_dy_knots"], dtype=np.float64).reshape(-1, order="F").copy()
    mp = np.ascontiguousarray(np.asarray(args["min_points_per_block"]).reshape(-1), dtype=np.int32)
    if mp.size < w:
        raise ValueError("min_points_per_block needs at least frame_w entries")
    keep = [t, xg, yg, frac, bx, by, bm, img, edx, edy, mp]
    flags = args["flags"].encode() if isinstance(args["flags"], str) else args["flags"]
    i = _In(flags, t.shape[0], t.shape[1], _ptr(t), _ptr(xg), _ptr(yg), hb, w, nF, _ptr(frac), _ptr(bx),
            _ptr(by), _ptr(bm), _ptr(img), _ptr(edx), _ptr(edy), _ptr(mp), int(args["group_size"]),
            int(args["max_iter"]), float(args["move_thresh"]), float(args["halt_correlation"]),
            float(args["correlation_increase_threshold"]), float(args["filter_strength"]),
            int(args["max_filter_iterations"]), float(args["filter_deactivation_threshold"]),
            float(args.get("lambda", 0.0)), float(args["linesearch_reduction_multiplier"]),
            int(args["solver_id"]), int(args["filter_id"]), int(n_threads))
    N = w * nF + 1
    mi = int(args["max_iter"])
    o = dict(p_last=np.zeros(2 * N), dx=np.zeros((w + 1) * nF), dy=np.zeros((w + 1) * nF),
             frame_corr=np.zeros(nF), residrms=np.zeros(nF), n_eval=np.zeros(nF, dtype=np.int64))
    if want_mask:
        o["mask_rm"] = np.zeros((hb, w * nF), dtype=np.uint8)
    if want_history:
        o["iter_corr"] = np.zeros(mi)
        o["frame_corr_hist"] = np.zeros((mi, nF))
        o["iter_errvals"] = np.zeros((2 * mi, nF))
        o["all_params"] = np.zeros((mi, 2 * N))
        o["rg_params"] = np.zeros((2 * mi, 2 * N))  # flag t: the chain after every half-step
    out = _Out(_ptr(o["p_last"]), _ptr(o["dx"]), _ptr(o["dy"]), _ptr(o["frame_corr"]), _ptr(o["residrms"]),
               _ptr(o["mask_rm"]) if want_mask else None,
               _ptr(o["iter_corr"]) if want_history else None,
               _ptr(o["frame_corr_hist"]) if want_history else None,
               _ptr(o["iter_errvals"]) if want_history else None,
               _ptr(o["all_params"]) if want_history else None,
               _ptr(o["n_eval"]), 0, 0, 0, _ptr(o["rg_params"]) if want_history else None)
    rc = L.sso_align_group(C.byref(i), C.byref(out))
    del keep
    if rc != 0:
        raise ValueError(f"oracle rejected the arguments (code {rc})")
    o["iterations"] = out.iterations
    o["stop_reason"] = out.stop_reason
    o["ls_trial_cap_hit"] = out.ls_trial_cap_hit
    if want_mask:
        o["mask"] = o.pop("mask_rm").astype(bool)  # frame_h x (W*nF), [row, col]
    return o


def smearing_filter(v, strength):
    a = np.ascontiguousarray(v, dtype=np.float64).copy()
    lib().sso_smearing_filter(_ptr(a), a.size, float(strength))
    return a


def range_filter(v, strength):
    a = np.ascontiguousarray(v, dtype=np.float64).copy()
    lib().sso_range_filter(_ptr(a), a.size, float(strength))
    return a


def organize2d1(px, py, n_frames, frame_w):
    px = np.ascontiguousarray(px, dtype=np.float64).reshape(-1, order="F")
    py = np.ascontiguousarray(py, dtype=np.float64).reshape(-1, order="F")
    p = np.zeros(2 * (frame_w * n_frames + 1))
    lib().sso_organize2d1(_ptr(px), _ptr(py), _ptr(p), n_frames, frame_w)
    return p


def organize1d2(p, n_frames, frame_w):
    p = np.ascontiguousarray(p, dtype=np.float64)
    px = np.zeros((frame_w + 1) * n_frames)
    py = np.zeros((frame_w + 1) * n_frames)
    lib().sso_organize1d2(_ptr(p), _ptr(px), _ptr(py), n_frames, frame_w)
    return px, py


def block_tridiag_solve(d, c, b):
    d = np.ascontiguousarray(d, dtype=np.float64)
    c = np.ascontiguousarray(c, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros_like(b)
    lib().sso_block_tridiag_solve(d.shape[0], _ptr(d), _ptr(c), _ptr(b), _ptr(x))
    return x


def _in_struct(args, n_threads=1):
    """sso_in for the 26 boundary arguments; returns (struct, keep-alive list)."""
    t = _rm(args["template_image"])
    xg = _rm(args["xgrad"])
    yg = _rm(args["ygrad"])
    frac = _rm(args["tfrac"])
    bx = _rm(args["basex"])
    by = _rm(args["basey"])
    bm = _rm(args["base_mask"], np.uint8)
    img = _rm(args["bmData"])
    nF = int(args["nFrames"])
    hb, w = frac.shape
    edx = np.asarray(args["est_dx_knots"], dtype=np.float64).reshape(-1, order="F").copy()
    edy = np.asarray(args["est_dy_knots"], dtype=np.float64).reshape(-1, order="F").copy()
    mp = np.ascontiguousarray(np.asarray(args["min_points_per_block"]).reshape(-1), dtype=np.int32)
    flags = args["flags"].encode() if isinstance(args["flags"], str) else bytes(args["flags"])
    keep = [t, xg, yg, frac, bx, by, bm, img, edx, edy, mp, flags]
    i = _In(flags, t.shape[0], t.shape[1], _ptr(t), _ptr(xg), _ptr(yg), hb, w, nF, _ptr(frac), _ptr(bx),
            _ptr(by), _ptr(bm), _ptr(img), _ptr(edx), _ptr(edy), _ptr(mp), int(args["group_size"]),
            int(args["max_iter"]), float(args["move_thresh"]), float(args["halt_correlation"]),
            float(args["correlation_increase_threshold"]), float(args["filter_strength"]),
            int(args["max_filter_iterations"]), float(args["filter_deactivation_threshold"]),
            float(args.get("lambda", 0.0)), float(args["linesearch_reduction_multiplier"]),
            int(args["solver_id"]), int(args["filter_id"]), int(n_threads))
    return i, keep


def debug_assemble(args: dict, p, shift: int) -> dict:
    """The reference's device state after one assembly pass at knot chain ``p`` (oracle hook)."""
    L = lib()
    L.sso_debug_assemble.argtypes = [C.c_void_p, C.c_void_p, C.c_int] + [C.c_void_p] * 15
    i, keep = _in_struct(args)
    hb, w = np.asarray(args["tfrac"]).shape
    nF = int(args["nFrames"])
    N = w * nF + 1
    npx = hb * w * nF
    spec = [("x", np.float64, npx), ("y", np.float64, npx), ("mask", np.uint8, npx), ("diff", np.float64, npx),
            ("wx", np.float64, npx), ("wy", np.float64, npx), ("params_used", np.uint8, N),
            ("blocks_present", np.uint8, N), ("offsets", np.int32, 2 * N), ("hv", np.float64, 12 * N),
            ("hr", np.int32, 12 * N), ("hc", np.int32, 12 * N), ("jtr", np.float64, 2 * N),
            ("errval", np.float64, 2 * nF)]
    o = {k: np.zeros(n, dt) for k, dt, n in spec}
    nu = C.c_int()
    pp = np.ascontiguousarray(p, dtype=np.float64)
    rc = L.sso_debug_assemble(C.byref(i), _ptr(pp), int(shift), *[_ptr(o[k]) for k, _, _ in spec], C.byref(nu))
    if rc != 0:
        raise ValueError(f"oracle rejected the arguments (code {rc})")
    o["n_used"] = nu.value
    del keep
    return o


def debug_expand(N, group_size, shift, params_used, offsets, new_delta_p, delta_p):
    L = lib()
    L.sso_debug_expand.argtypes = [C.c_int, C.c_int, C.c_int] + [C.c_void_p] * 4
    pu = np.ascontiguousarray(params_used, dtype=np.uint8)
    off = np.ascontiguousarray(offsets, dtype=np.int32)
    nd = np.ascontiguousarray(new_delta_p, dtype=np.float64)
    d = np.ascontiguousarray(delta_p, dtype=np.float64).copy()
    L.sso_debug_expand(int(N), int(group_size), int(shift), _ptr(pu), _ptr(off), _ptr(nd), _ptr(d))
    return d


def debug_global_corr(args, mask, diff):
    L = lib()
    L.sso_debug_global_corr.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.sso_debug_global_corr.restype = C.c_double
    i, keep = _in_struct(args)
    m = np.ascontiguousarray(mask, dtype=np.uint8).reshape(-1)
    d = np.ascontiguousarray(diff, dtype=np.float64).reshape(-1)
    r = L.sso_debug_global_corr(C.byref(i), _ptr(m), _ptr(d))
    del keep
    return r
