"""ctypes binding of libsteadyscan_b200.so (the C ABI of include/steadyscan_b200.h)."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsteadyscan_b200.so")

SS_F64, SS_F32, SS_U16, SS_F16, SS_U8, SS_I32 = 0, 1, 2, 3, 4, 5
SS_HOST, SS_DEVICE = 0, 1
STATUS = {0: "SS_OK", -1: "SS_ERR_INVALID_ARGUMENT", -2: "SS_ERR_CUDA", -3: "SS_ERR_OUT_OF_MEMORY",
          -4: "SS_ERR_NO_DEVICE", -5: "SS_ERR_BUSY", -6: "SS_ERR_NOT_FOUND"}
STOP_NAMES = ["CorrelationIncreaseThreshold", "HaltCorrelation", "MovementThreshold", "IterationLimit", "Error"]


class SSMatrix(C.Structure):
    _fields_ = [("data", C.c_void_p), ("rows", C.c_int64), ("cols", C.c_int64), ("dtype", C.c_int32),
                ("location", C.c_int32)]


class SSInputs(C.Structure):
    _fields_ = [
        ("flags", C.c_char_p),
        ("template_image", SSMatrix), ("xgrad", SSMatrix), ("ygrad", SSMatrix), ("tfrac", SSMatrix),
        ("basex", SSMatrix), ("basey", SSMatrix), ("base_mask", SSMatrix), ("bm_data", SSMatrix),
        ("est_dx_knots", SSMatrix), ("est_dy_knots", SSMatrix),
        ("group_size", C.c_int32), ("n_frames", C.c_int32), ("min_points_per_block", SSMatrix),
        ("max_iter", C.c_int32), ("move_thresh", C.c_double), ("halt_correlation", C.c_double),
        ("correlation_increase_threshold", C.c_double), ("filter_strength", C.c_double),
        ("max_filter_iterations", C.c_int32), ("filter_deactivation_threshold", C.c_double),
        ("lam", C.c_double), ("linesearch_reduction_multiplier", C.c_double), ("solver_id", C.c_int32),
        ("filter_id", C.c_int32), ("gpu_device_id", C.c_int32), ("template_storage", C.c_int32),
        ("frames_per_cta", C.c_int32),
    ]


class SSOutputs(C.Structure):
    _fields_ = [
        ("dx_knots", C.c_void_p), ("dy_knots", C.c_void_p), ("frame_corr", C.c_void_p), ("iter_used", C.c_void_p),
        ("mask", C.c_void_p), ("residrms", C.c_void_p), ("device_init_time", C.c_void_p),
        ("iteration_corr", C.c_void_p), ("frame_corr_history", C.c_void_p), ("iteration_errvals", C.c_void_p),
        ("raw_params", C.c_void_p), ("all_params", C.c_void_p), ("frame_params", C.c_void_p),
        ("stop_reason", C.c_int32), ("trial_cap_hit", C.c_int32), ("n_frame_passes", C.c_int64),
        ("elapsed_ms", C.c_double), ("blocks_used", C.c_void_p),
        ("iteration_times", C.c_void_p), ("function_times", C.c_void_p), ("rg_params", C.c_void_p),
    ]


class SSRecording(C.Structure):
    _fields_ = [("group", SSInputs), ("frames_per_set", C.c_int32), ("min_frames_per_set", C.c_int32),
                ("corr_thresh", C.c_double), ("minblockfrac", C.c_double), ("per_set_estimates", C.c_int32)]


class SSRecordingOutputs(C.Structure):
    _fields_ = [("dx_knots", C.c_void_p), ("dy_knots", C.c_void_p), ("corr", C.c_void_p), ("iter_used", C.c_void_p),
                ("residrms", C.c_void_p), ("failed", C.c_void_p), ("blocks_used", C.c_void_p),
                ("n_sets", C.c_int32)]


class SSPrepFrames(C.Structure):
    _fields_ = [("frames", SSMatrix), ("n_frames", C.c_int32), ("pregauss", C.c_double), ("mednorm", C.c_int32),
                ("cropping", C.c_int32 * 4), ("gather", C.c_void_p), ("block_h", C.c_int32), ("n_blocks", C.c_int32),
                ("out", SSMatrix), ("gpu_device_id", C.c_int32)]


class SSReconstruct(C.Structure):
    _fields_ = [("frames", SSMatrix), ("n_frames", C.c_int32), ("basex", SSMatrix), ("basey", SSMatrix),
                ("tfrac", SSMatrix), ("prevknotind", SSMatrix), ("dx_knots", SSMatrix), ("dy_knots", SSMatrix),
                ("template_h", C.c_int32), ("template_w", C.c_int32), ("regfac", C.c_double),
                ("pixel_aspect_ratio", C.c_double), ("out", SSMatrix), ("mask", C.c_void_p),
                ("iterations", C.c_void_p), ("gpu_device_id", C.c_int32)]


class SSBatchStats(C.Structure):
    _fields_ = [("n_groups", C.c_int32), ("cycles", C.c_int32), ("linesearch_rounds", C.c_int32),
                ("kernel_launches", C.c_int32), ("frame_passes", C.c_int64 * 4), ("eval_ms", C.c_double * 4),
                ("arena_bytes", C.c_int64), ("run_ms", C.c_double), ("staging", C.c_int64 * 6),
                ("assembly_columns_kept", C.c_int64)]


_lib = None


def load(build_if_missing: bool = True):
    """Loads the CUDA library; raises if it is missing (there is no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        if not build_if_missing:
            raise ImportError(f"{LIB_PATH} is missing; build it with python -m steadyscan_b200.build")
        from . import build as _build
        _build.build()
    lib = C.CDLL(LIB_PATH)
    lib.ss_align_group_to_template.argtypes = [C.POINTER(SSInputs), C.POINTER(SSOutputs)]
    lib.ss_align_group_to_template.restype = C.c_int
    lib.ss_align_groups.argtypes = [C.c_int32, C.POINTER(SSInputs), C.POINTER(SSOutputs)]
    lib.ss_align_groups.restype = C.c_int
    lib.ss_last_error.argtypes = []
    lib.ss_last_error.restype = C.c_char_p
    lib.ss_abi_version.argtypes = []
    lib.ss_abi_version.restype = C.c_int32
    lib.ss_batch_create.argtypes = [C.c_int32, C.POINTER(SSInputs), C.POINTER(SSOutputs), C.POINTER(C.c_void_p)]
    lib.ss_batch_create.restype = C.c_int
    for name in ("ss_batch_run", "ss_batch_collect"):
        getattr(lib, name).argtypes = [C.c_void_p]
        getattr(lib, name).restype = C.c_int
    lib.ss_batch_set_timing.argtypes = [C.c_void_p, C.c_int32]
    lib.ss_batch_set_timing.restype = C.c_int
    lib.ss_batch_set_graph.argtypes = [C.c_void_p, C.c_int32]
    lib.ss_batch_set_graph.restype = C.c_int
    lib.ss_batch_stats_get.argtypes = [C.c_void_p, C.POINTER(SSBatchStats)]
    lib.ss_batch_stats_get.restype = C.c_int
    lib.ss_batch_stream.argtypes = [C.c_void_p]
    lib.ss_batch_stream.restype = C.c_void_p
    lib.ss_batch_destroy.argtypes = [C.c_void_p]
    lib.ss_batch_destroy.restype = None
    lib.ss_session_create.argtypes = [C.POINTER(SSInputs), C.POINTER(C.c_void_p)]
    lib.ss_session_create.restype = C.c_int
    lib.ss_session_destroy.argtypes = [C.c_void_p]
    lib.ss_session_destroy.restype = None
    lib.ss_batch_measure.argtypes = [C.c_int32, C.POINTER(SSInputs), C.POINTER(SSOutputs), C.c_void_p,
                                     C.POINTER(C.c_int64)]
    lib.ss_batch_measure.restype = C.c_int
    lib.ss_batch_create_ex.argtypes = [C.c_int32, C.POINTER(SSInputs), C.POINTER(SSOutputs), C.c_void_p,
                                       C.c_void_p, C.c_int64, C.POINTER(C.c_void_p)]
    lib.ss_batch_create_ex.restype = C.c_int
    for name in ("ss_batch_start", "ss_batch_step", "ss_batch_poll"):
        getattr(lib, name).argtypes = [C.c_void_p]
        getattr(lib, name).restype = C.c_int
    lib.ss_server_create.argtypes = [C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]
    lib.ss_server_create.restype = C.c_int
    lib.ss_server_admit.argtypes = [C.c_void_p, C.POINTER(SSInputs), C.POINTER(SSOutputs), C.c_void_p, C.c_void_p,
                                    C.c_int64, C.POINTER(C.c_int32)]
    lib.ss_server_admit.restype = C.c_int
    lib.ss_server_step.argtypes = [C.c_void_p]
    lib.ss_server_step.restype = C.c_int
    lib.ss_server_poll.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.c_int32, C.POINTER(C.c_int32)]
    lib.ss_server_poll.restype = C.c_int
    lib.ss_server_active.argtypes = [C.c_void_p]
    lib.ss_server_active.restype = C.c_int32
    lib.ss_server_destroy.argtypes = [C.c_void_p]
    lib.ss_server_destroy.restype = None
    lib.ss_solve_block_tridiagonal.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                               C.c_void_p]
    lib.ss_solve_block_tridiagonal.restype = C.c_int
    lib.ss_solve_block_tridiagonal_noalloc.argtypes = [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                       C.c_void_p]
    lib.ss_solve_block_tridiagonal_noalloc.restype = C.c_int
    lib.ss_estimate_displacements.argtypes = [C.POINTER(SSRecording), C.POINTER(SSRecordingOutputs)]
    lib.ss_estimate_displacements.restype = C.c_int
    lib.ss_recording_sets.argtypes = [C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                      C.c_int32, C.POINTER(C.c_int32)]
    lib.ss_recording_sets.restype = C.c_int
    lib.ss_prepare_frames.argtypes = [C.POINTER(SSPrepFrames)]
    lib.ss_prepare_frames.restype = C.c_int
    lib.ss_reconstruct_frames.argtypes = [C.POINTER(SSReconstruct)]
    lib.ss_reconstruct_frames.restype = C.c_int
    _lib = lib
    return lib


class SteadyScanError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{STATUS.get(code, code)}: {message}")
        self.code = code


def check(rc: int):
    if rc != 0:
        raise SteadyScanError(rc, load().ss_last_error().decode(errors="replace"))
