"""Host logic of the recording-level estimate, without a GPU: the library's set split
(ss_recording_sets) against the restatement of steady_scan.m:97-108 / :216-220, and the
post-estimate rules of the restatement on hand-made cases (steady_scan.m:246-284, :615-623)."""
import numpy as np
import pytest

from oracle import estimate
from steadyscan_b200 import api


@pytest.mark.parametrize("n,fps,minfps", [(1, 500, 100), (2, 500, 100), (11, 4, 2), (12, 4, 2), (13, 4, 3),
                                          (1000, 500, 100), (1050, 500, 100), (1001, 500, 100), (17, 5, 0),
                                          (9, 3, 5), (4000, 500, 100), (64, 64, 10), (65, 64, 10)])
def test_set_split_matches_restatement(n, fps, minfps):
    assert api.recording_sets(n, fps, minfps) == estimate.sets(n, fps, minfps)


def test_set_split_by_hand():
    # 11 frames, sets of 4: [1..5], [5..9], [9..11] (1-based, overlap frame included)
    assert estimate.sets(11, 4, 2) == [(0, 5), (4, 5), (8, 3)]
    # the rebalancing of the last two set sizes (1002 frames: 500, 500, 2 -> 500, 251, 251) moves no
    # frame, because the loop reads the unchanged set starts
    start, size = estimate.set_starts(1002, 500, 100)
    assert size == [500, 251, 251]
    assert estimate.sets(1002, 500, 100) == [(0, 501), (500, 501), (1000, 2)]
    # one frame: a set of one frame keeps no frame (the overlap frame is dropped)
    assert estimate.sets(1, 500, 100) == [(0, 1)]


def test_set_split_rejects_bad_arguments():
    with pytest.raises(api.SteadyScanError):
        api.recording_sets(0, 500, 100)
    with pytest.raises(api.SteadyScanError):
        api.recording_sets(10, 0, 100)


def test_extend_firstandlast_by_hand():
    x = np.array([1.0, 2.0, 3.0, 4.0, 5.0, 6.0])
    # blocks 2..3 (0-based) used of 5: knots 0-1 take knot 2, knots 4-5 take knot 3
    np.testing.assert_array_equal(estimate.extend_firstandlast(x, [0, 0, 1, 1, 0]), [3, 3, 3, 4, 4, 4])
    # the function rewrites the knots after the last used block even when every block is used (the
    # caller only calls it when the first or the last block is unused)
    np.testing.assert_array_equal(estimate.extend_firstandlast(x, [1, 1, 1, 1, 1]), [1, 2, 3, 4, 5, 5])
    np.testing.assert_array_equal(estimate.extend_firstandlast(x, [0, 0, 0, 0, 0]), x)
    np.testing.assert_array_equal(estimate.extend_firstandlast(x, [1, 0, 0, 0, 0]), [1, 1, 1, 1, 1, 1])
