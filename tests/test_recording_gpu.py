"""ss_estimate_displacements (the reference driver's estimate loop over a recording, with the
post-estimate validity rules on the device) against the CPU restatement of steady_scan.m:157-288
over the FP64 oracle, through the C ABI.

The recording has 11 frames in sets of 4 (sets of 5, 5 and 3 frames with their overlap frames), so
the recording's last frame is never estimated (NaN). Its first frame starts 500 px off the template
(no block is ever used: failed, NaN correlation); as the reference passes the whole estimate matrix
to every set, every set starts from the recording's first columns, so each set's first frame does
the same. Its second frame starts with its first knots 60 px above the template, so its first
blocks stay unused and extend_firstandlast repeats the first used block's knots."""
import numpy as np
import pytest

from oracle import estimate
from steadyscan_b200 import api
from tests.helpers import make_args

pytestmark = pytest.mark.gpu


def _recording(seed=91, n_frames=11):
    args, _, s = make_args(n_frames=n_frames, seed=seed, frame_dtype=np.uint16)
    ex = np.zeros_like(args["est_dx_knots"])
    ey = np.zeros_like(args["est_dy_knots"])
    ex[:, 0] = 500.0
    ey[:3, 1] = -60.0
    args["est_dx_knots"] = ex
    args["est_dy_knots"] = ey
    return args, s


def _compare(g, o, knot_tol):
    assert g["n_sets"] == o["n_sets"]
    np.testing.assert_array_equal(g["failed"], o["failed"])
    np.testing.assert_array_equal(g["blocks_used"], o["blocks_used"])
    np.testing.assert_array_equal(np.isnan(g["dx_knots"]), np.isnan(o["dx_knots"]))
    np.testing.assert_allclose(g["dx_knots"], o["dx_knots"], atol=knot_tol, rtol=0, equal_nan=True)
    np.testing.assert_allclose(g["dy_knots"], o["dy_knots"], atol=knot_tol, rtol=0, equal_nan=True)
    np.testing.assert_array_equal(g["iter_used"], o["iter_used"])
    np.testing.assert_allclose(g["corr"], o["corr"], atol=1e-9, rtol=1e-9, equal_nan=True)
    np.testing.assert_allclose(g["residrms"], o["residrms"], atol=1e-9, rtol=1e-9, equal_nan=True)


@pytest.mark.parametrize("per_set", [False, True])
def test_estimate_displacements_matches_restatement(per_set):
    args, s = _recording()
    kw = dict(frames_per_set=4, min_frames_per_set=2, corr_thresh=s["corr_thresh"], minblockfrac=s["minblockfrac"],
              per_set_estimates=per_set)
    o = estimate.estimate_displacements(args, **kw)
    g = api.estimate_displacements(args, **kw)
    _compare(g, o, 1e-6)
    # the cases the recording was built for
    assert np.isnan(g["dx_knots"][:, -1]).all() and np.isnan(g["corr"][-1]) and not g["failed"][-1]
    assert g["failed"][0] and np.isnan(g["corr"][0])
    if not per_set:
        assert g["failed"][4] and g["failed"][8]  # each set starts from the recording's first columns
    assert not g["blocks_used"][0, 1]
    np.testing.assert_array_equal(g["dy_knots"][0, 1], g["dy_knots"][int(np.argmax(g["blocks_used"][:, 1])), 1])


def test_estimate_displacements_equals_per_set_group_calls():
    """Every kept frame's knots equal those of its set run alone through align_group_to_template."""
    args, s = _recording(seed=92, n_frames=9)
    g = api.estimate_displacements(args, frames_per_set=4, min_frames_per_set=2)
    w = args["tfrac"].shape[1]
    for first, count in api.recording_sets(9, 4, 2):
        a = dict(args)
        a["bmData"] = np.asfortranarray(args["bmData"][:, first * w:(first + count) * w])
        a["nFrames"] = count
        a["est_dx_knots"] = args["est_dx_knots"][:, :count]
        a["est_dy_knots"] = args["est_dy_knots"][:, :count]
        r = api.align_group(a)
        for j in range(count - 1):
            if g["failed"][first + j] and np.isnan(g["corr"][first + j]):
                continue
            if g["blocks_used"][:, first + j].all():
                np.testing.assert_array_equal(g["dx_knots"][:, first + j], r["dx"].reshape(count, w + 1)[j])
            np.testing.assert_array_equal(g["blocks_used"][:, first + j], r["blocks_used"][:, j])


def test_precision_s_recording_within_bound():
    args, s = _recording(seed=93)
    o = estimate.estimate_displacements(args, frames_per_set=4, min_frames_per_set=2)
    g = api.estimate_displacements(dict(args, flags="S"), frames_per_set=4, min_frames_per_set=2)
    ok = ~np.isnan(o["dx_knots"][0]) & ~o["failed"] & ~g["failed"]
    d = np.concatenate([(g["dx_knots"] - o["dx_knots"])[:, ok].ravel(), (g["dy_knots"] - o["dy_knots"])[:, ok].ravel()])
    assert ok.any()
    assert float(np.sqrt(np.mean(d * d))) <= 0.02
