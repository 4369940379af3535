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
