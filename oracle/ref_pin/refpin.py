"""ctypes front of oracle/_ref/libssref.so: the reference's own device functions and host classes,
host-compiled (see ref_wrap.cpp). TEST INFRASTRUCTURE ONLY; needs the reference tree to build."""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.abspath(os.path.join(HERE, "..", "_ref", "libssref.so"))
REF_TREE = os.environ.get("STEADYSCAN_REFERENCE_SOURCE", "/root/reference/setup/source")
_lib = None


class State(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("frame_h", "frame_w", "n_frames", "templ_h", "templ_w", "group_size")] + \
        [(n, C.c_void_p) for n in ("templ", "xgrad", "ygrad", "frac", "basex", "basey", "image", "base_mask",
                                   "min_points", "p", "x", "y", "diff", "wx", "wy", "jtr", "errval", "hv",
                                   "delta_p", "new_delta_p", "mask", "params_used", "blocks_present",
                                   "group_active", "offsets", "hr", "hc")] + [("n_used", C.c_int)]


def available() -> bool:
    return os.path.exists(LIB) or os.path.isdir(REF_TREE)


def build() -> str:
    if not os.path.exists(LIB):
        subprocess.check_call(["make", "-s", "-C", HERE])
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(LIB)
        _lib.ssref_assemble.argtypes = [C.POINTER(State), C.c_int]
        _lib.ssref_expand.argtypes = [C.POINTER(State), C.c_int]
        _lib.ssref_global_corr.argtypes = [C.POINTER(State)]
        _lib.ssref_global_corr.restype = C.c_double
        _lib.ssref_organize2d1.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        _lib.ssref_organize1d2.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        _lib.ssref_smearing_filter.argtypes = [C.c_void_p, C.c_int, C.c_double]
        _lib.ssref_range_filter.argtypes = [C.c_void_p, C.c_int, C.c_double]
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def make_state(args: dict, p: np.ndarray):
    """Reference device state for the 26 boundary arguments (row-major, as NeutralMatrix RowMajor)."""
    rm = lambda a, dt=np.float64: np.ascontiguousarray(np.asarray(a, dtype=dt))
    frac = rm(args["tfrac"])
    hb, w = frac.shape
    nF = int(args["nFrames"])
    fW, N = w * nF, w * nF + 1
    npx = hb * fW
    gs = int(args["group_size"])
    ng = fW // gs
    arrs = dict(templ=rm(args["template_image"]), xgrad=rm(args["xgrad"]), ygrad=rm(args["ygrad"]), frac=frac,
                basex=rm(args["basex"]), basey=rm(args["basey"]), image=rm(args["bmData"]),
                base_mask=rm(args["base_mask"], np.uint8),
                min_points=np.ascontiguousarray(np.asarray(args["min_points_per_block"]).reshape(-1), dtype=np.int32),
                p=np.ascontiguousarray(p, dtype=np.float64).copy(), x=np.zeros(npx), y=np.zeros(npx),
                diff=np.zeros(npx), wx=np.zeros(npx), wy=np.zeros(npx), jtr=np.zeros(2 * N),
                errval=np.full(2 * nF, 1e6), hv=np.zeros(12 * N), delta_p=np.zeros(2 * N),
                new_delta_p=np.zeros(2 * N), mask=np.zeros(npx, np.uint8), params_used=np.zeros(N, np.uint8),
                blocks_present=np.zeros(N, np.uint8), group_active=np.ones(2 * ng + 64, np.uint8),
                offsets=np.zeros(2 * N, np.int32), hr=np.zeros(12 * N, np.int32), hc=np.zeros(12 * N, np.int32))
    arrs["group_active"][2 * ng:] = 0
    st = State(hb, w, nF, arrs["templ"].shape[0], arrs["templ"].shape[1], gs,
               *[_p(arrs[n]) for n in ("templ", "xgrad", "ygrad", "frac", "basex", "basey", "image", "base_mask",
                                      "min_points", "p", "x", "y", "diff", "wx", "wy", "jtr", "errval", "hv",
                                      "delta_p", "new_delta_p", "mask", "params_used", "blocks_present",
                                      "group_active", "offsets", "hr", "hc")], 0)
    return st, arrs


def assemble(args: dict, p: np.ndarray, shift: int):
    st, a = make_state(args, p)
    lib().ssref_assemble(C.byref(st), int(shift))
    a["n_used"] = st.n_used
    return a


def expand(args, p, shift, params_used, offsets, new_delta_p, delta_p):
    st, a = make_state(args, p)
    a["params_used"][:] = params_used
    a["offsets"][:] = offsets
    a["new_delta_p"][:] = new_delta_p
    a["delta_p"][:] = delta_p
    lib().ssref_expand(C.byref(st), int(shift))
    return a["delta_p"]


def global_corr(args, mask, diff):
    st, a = make_state(args, np.zeros(2 * (int(args["nFrames"]) * args["tfrac"].shape[1] + 1)))
    a["mask"][:] = np.asarray(mask, np.uint8).reshape(-1)
    a["diff"][:] = np.asarray(diff, np.float64).reshape(-1)
    return lib().ssref_global_corr(C.byref(st)), a["diff"]


def organize2d1(px, py, n_frames, frame_w):
    px = np.ascontiguousarray(px, dtype=np.float64).reshape(-1, order="F").copy()
    py = np.ascontiguousarray(py, dtype=np.float64).reshape(-1, order="F").copy()
    p = np.zeros(2 * (frame_w * n_frames + 1))
    lib().ssref_organize2d1(_p(px), _p(py), _p(p), n_frames, frame_w)
    return p


def organize1d2(p, n_frames, frame_w):
    p = np.ascontiguousarray(p, dtype=np.float64).copy()
    px = np.zeros((frame_w + 1) * n_frames)
    py = np.zeros((frame_w + 1) * n_frames)
    lib().ssref_organize1d2(_p(p), _p(px), _p(py), n_frames, frame_w)
    return px, py


def smearing_filter(v, strength):
    a = np.ascontiguousarray(v, dtype=np.float64).copy()
    lib().ssref_smearing_filter(_p(a), a.size, float(strength))
    return a


def range_filter(v, strength):
    a = np.ascontiguousarray(v, dtype=np.float64).copy()
    lib().ssref_range_filter(_p(a), a.size, float(strength))
    return a


# ------------------------------------------------------------------------------------------------
# The reference's whole task layer on the host (oracle/_ref/libssrefrun.so, refrun.cpp)

RUN_LIB = os.path.abspath(os.path.join(HERE, "..", "_ref", "libssrefrun.so"))
_run_lib = None


class RunIn(C.Structure):
    _fields_ = [("flags", C.c_char_p), ("templ_h", C.c_int), ("templ_w", C.c_int), ("templ", C.c_void_p),
                ("xgrad", C.c_void_p), ("ygrad", C.c_void_p), ("frame_h", C.c_int), ("frame_w", C.c_int),
                ("n_frames", C.c_int), ("frac", C.c_void_p), ("basex", C.c_void_p), ("basey", C.c_void_p),
                ("base_mask", C.c_void_p), ("image", C.c_void_p), ("est_dx", C.c_void_p), ("est_dy", C.c_void_p),
                ("min_points", C.c_void_p), ("group_size", C.c_int), ("max_iter", C.c_int),
                ("move_thresh", C.c_double), ("halt_corr", C.c_double), ("corr_inc_thresh", C.c_double),
                ("filter_strength", C.c_double), ("max_filter_iter", C.c_int), ("filter_corr_thresh", C.c_double),
                ("lam", C.c_double), ("ls_mult", C.c_double), ("solver_id", C.c_int), ("filter_id", C.c_int)]


class RunOut(C.Structure):
    _fields_ = [("dx", C.c_void_p), ("dy", C.c_void_p), ("frame_corr", C.c_void_p), ("residrms", C.c_void_p),
                ("mask", C.c_void_p), ("all_params", C.c_void_p), ("iter_errvals", C.c_void_p),
                ("iter_corr", C.c_void_p), ("frame_corr_hist", C.c_void_p), ("iterations", C.c_int),
                ("stop_reason", C.c_int), ("singular_solves", C.c_int), ("rg_params", C.c_void_p)]


def run_available() -> bool:
    return os.path.exists(RUN_LIB) or os.path.isdir(REF_TREE)


def run_lib():
    global _run_lib
    if _run_lib is None:
        if not os.path.exists(RUN_LIB):
            subprocess.check_call(["make", "-s", "-C", HERE])
        _run_lib = C.CDLL(RUN_LIB)
        _run_lib.ssrun_align.argtypes = [C.POINTER(RunIn), C.POINTER(RunOut)]
        _run_lib.ssrun_align.restype = C.c_int
    return _run_lib


def run_align(args: dict) -> dict:
    """The reference's align_group_to_template task (Task::alignFrames with MainIteration, its
    kernels and filters, solver id 1) on the 26 boundary arguments; returns its outputs: knots,
    frame correlations, residrms, mask, the knot chain after every iteration (all_params) and, with
    flags e / C, the errvals of every half-step and the global correlation of every iteration, and with
    flag t the chain after every half-step (rg_params, 2 max_iter x 2N; NaN without flag t)."""
    rm = lambda a, dt=np.float64: np.ascontiguousarray(np.asarray(a, dtype=dt))
    t, xg, yg = rm(args["template_image"]), rm(args["xgrad"]), rm(args["ygrad"])
    frac, bx, by = rm(args["tfrac"]), rm(args["basex"]), rm(args["basey"])
    bm, img = rm(args["base_mask"], np.uint8), rm(args["bmData"])
    hb, w = frac.shape
    nF = int(args["nFrames"])
    edx = np.asarray(args["est_dx_knots"], dtype=np.float64).reshape(-1, order="F").copy()
    edy = np.asarray(args["est_dy_knots"], dtype=np.float64).reshape(-1, order="F").copy()
    mp = np.ascontiguousarray(np.asarray(args["min_points_per_block"]).reshape(-1)[:w], dtype=np.int32)
    flags = args["flags"].encode() if isinstance(args["flags"], str) else bytes(args["flags"])
    mi = int(args["max_iter"])
    N = w * nF + 1
    keep = [t, xg, yg, frac, bx, by, bm, img, edx, edy, mp, flags]
    i = RunIn(flags, t.shape[0], t.shape[1], _p(t), _p(xg), _p(yg), hb, w, nF, _p(frac), _p(bx), _p(by), _p(bm),
              _p(img), _p(edx), _p(edy), _p(mp), int(args["group_size"]), mi, float(args["move_thresh"]),
              float(args["halt_correlation"]), float(args["correlation_increase_threshold"]),
              float(args["filter_strength"]), int(args["max_filter_iterations"]),
              float(args["filter_deactivation_threshold"]), float(args.get("lambda", 0.0)),
              float(args["linesearch_reduction_multiplier"]), int(args["solver_id"]), int(args["filter_id"]))
    o = dict(dx=np.zeros((w + 1) * nF), dy=np.zeros((w + 1) * nF), frame_corr=np.zeros(nF), residrms=np.zeros(nF),
             mask=np.zeros((hb, w * nF), np.uint8), all_params=np.zeros((mi, 2 * N)),
             iter_errvals=np.zeros((nF, 2 * mi)), iter_corr=np.zeros(mi), frame_corr_hist=np.zeros((mi, nF)),
             rg_params=np.full((2 * mi, 2 * N), np.nan))
    out = RunOut(*[_p(o[k]) for k in ("dx", "dy", "frame_corr", "residrms", "mask", "all_params", "iter_errvals",
                                      "iter_corr", "frame_corr_hist")], 0, 0, 0, _p(o["rg_params"]))
    rc = run_lib().ssrun_align(C.byref(i), C.byref(out))
    del keep
    if rc != 0:
        raise RuntimeError(f"reference run failed ({rc})")
    o["iterations"] = out.iterations
    o["stop_reason"] = out.stop_reason
    o["singular_solves"] = out.singular_solves
    o["mask"] = o["mask"].astype(bool)
    o["iter_errvals"] = o["iter_errvals"].T.copy()  # (2 max_iter) x nF, as the MEX output
    return o
