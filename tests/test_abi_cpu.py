"""The C-ABI library on a machine without a GPU: it loads, exports every declared entry point, and
rejects malformed arguments with the reference's error semantics before any device work."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from steadyscan_b200 import _lib, api, build
from tests.helpers import make_args

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _lib.load()


def declared_symbols():
    names = []
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            names += re.findall(r"SS_API\s+[\w\s\*]+?\b(ss_\w+)\s*\(", text)
    return names


def test_exports_every_declared_symbol(lib):
    names = declared_symbols()
    assert "ss_align_group_to_template" in names and "ss_align_groups" in names
    for n in names:
        assert hasattr(lib, n), f"{n} not exported"


def test_abi_version(lib):
    assert lib.ss_abi_version() == 6  # outputs 9, 10 and 14 (flags T and t) at the end of ss_outputs


def test_struct_sizes_match_header(lib):
    """The ctypes mirrors have the C structs' layout: the last field sits where the header puts it."""
    assert C.sizeof(_lib.SSOutputs) == 13 * 8 + 4 + 4 + 8 + 8 + 8 + 3 * 8
    assert _lib.SSOutputs.rg_params.offset == 13 * 8 + 4 + 4 + 8 + 8 + 8 + 2 * 8
    assert _lib.SSRecording.corr_thresh.offset == C.sizeof(_lib.SSInputs) + 8
    assert C.sizeof(_lib.SSRecordingOutputs) == 7 * 8 + 8
    # ss_prep_frames: ss_matrix (32), n_frames (+pad), pregauss at 40, mednorm 48, cropping 52..68,
    # gather at 72, block_h/n_blocks, out at 88, gpu_device_id at 120, padded to 128
    assert _lib.SSPrepFrames.pregauss.offset == 40
    assert _lib.SSPrepFrames.gather.offset == 72
    assert _lib.SSPrepFrames.out.offset == 88
    assert C.sizeof(_lib.SSPrepFrames) == 128
    # ss_reconstruct: frames, n_frames (+pad), six matrices from 40, template_h/w at 232, regfac 240,
    # aspect 248, out 256, mask 288, iterations 296, gpu_device_id 304, padded to 312
    assert _lib.SSReconstruct.basex.offset == 40
    assert _lib.SSReconstruct.template_h.offset == 232
    assert _lib.SSReconstruct.out.offset == 256
    assert _lib.SSReconstruct.gpu_device_id.offset == 304
    assert C.sizeof(_lib.SSReconstruct) == 312


def _expect_invalid(args, match):
    with pytest.raises(api.SteadyScanError) as e:
        api.align_group(args)
    assert e.value.code == -1
    assert re.search(match, str(e.value))


def test_rejects_missing_precision(lib):
    args, _, _ = make_args(nlines=16, linewidth=12, nknots=5, n_frames=2)
    args["flags"] = "C"
    _expect_invalid(args, "precision")


def test_rejects_bad_solver_and_filter(lib):
    args, _, _ = make_args(nlines=16, linewidth=12, nknots=5, n_frames=2)
    args["solver_id"] = 3
    _expect_invalid(args, "solver")
    args["solver_id"] = 2
    args["filter_id"] = 7
    _expect_invalid(args, "filter")
    args["max_filter_iterations"] = 0  # the filter factory ignores the id then (task.cpp:54)
    try:
        api.align_group(args)  # passes validation; on a machine without a GPU it stops at the device
    except api.SteadyScanError as e:
        assert e.code == -4, str(e)


def test_rejects_shape_mismatch(lib):
    args, _, _ = make_args(nlines=16, linewidth=12, nknots=5, n_frames=2)
    args["bmData"] = args["bmData"][:, :-1]
    _expect_invalid(args, "bm_data")
    args, _, _ = make_args(nlines=16, linewidth=12, nknots=5, n_frames=2)
    args["group_size"] = args["tfrac"].shape[1] + 1
    _expect_invalid(args, "group_size")
    args, _, _ = make_args(nlines=16, linewidth=12, nknots=5, n_frames=2)
    args["xgrad"] = args["xgrad"][:, :-1]
    _expect_invalid(args, "xgrad")


def test_not_enough_inputs(lib):
    with pytest.raises(api.SteadyScanError) as e:
        api.align_group_to_template("D", np.zeros((4, 4)))
    assert "expected 26" in str(e.value)
