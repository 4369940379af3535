"""The caller-side preparation of the boundary inputs (prep.py) against values worked out by hand
from steady_scan.m:748-828 (init_settings: scan times, knot times, tfrac, basex/basey),
:601-613 (image2blockmatrix), :174-175 (min_points_per_block) and :177-179 (gradients)."""
import numpy as np

from steadyscan_b200 import prep


def test_uniform_two_lines_per_knot():
    # 4 lines x 3 pixels, 3 knots: 12 pixels, dwell 1/12, scan time 1/24 + (3 l + j) / 12; knots at
    # the first pixel of lines 0 and 2: t = [0, 1/2, 1]
    tmpl = np.zeros((4, 3))
    s = prep.init_settings({"nknots": 3}, tmpl, 4, 3)
    np.testing.assert_allclose(s["t_knots"], [0.0, 0.5, 1.0], rtol=0, atol=1e-15)
    np.testing.assert_array_equal(s["prevknotind"], [[1, 1, 1], [1, 1, 1], [2, 2, 2], [2, 2, 2]])
    l, j = np.mgrid[0:4, 0:3]
    np.testing.assert_allclose(s["tfrac"], 1 / 12 + ((l % 2) * 3 + j) / 6, rtol=0, atol=1e-15)
    # template of the data's size: subrec [1 3 1 4], basex = j + 1, basey = l + 1 (1-based)
    np.testing.assert_array_equal(s["basex"], j + 1)
    np.testing.assert_array_equal(s["basey"], l + 1)
    lay = prep.block_layout(s)
    assert (lay.frame_h, lay.frame_w) == (6, 2)
    # block 1 holds lines 0-1 in column-major order: (0,0) (1,0) (0,1) (1,1) (0,2) (1,2)
    np.testing.assert_allclose(lay.tfrac[:, 0], np.array([1, 7, 3, 9, 5, 11]) / 12, rtol=0, atol=1e-15)
    np.testing.assert_array_equal(lay.basex[:, 0], [0, 0, 1, 1, 2, 2])
    np.testing.assert_array_equal(lay.basey[:, 0], [0, 1, 0, 1, 0, 1])
    np.testing.assert_array_equal(lay.basey[:, 1], [2, 3, 2, 3, 2, 3])
    assert lay.base_mask.all()
    # histc(prevknotind, 1:3) = [6 6 0], times 0.3, truncated
    np.testing.assert_array_equal(lay.min_points, [1, 1, 0])
    # the frame in block order follows the same gather
    frame = np.arange(12, dtype=np.float64).reshape(4, 3)
    bm = prep.frames_to_blockmatrix(frame, lay)
    np.testing.assert_array_equal(bm[:, 0], [frame[0, 0], frame[1, 0], frame[0, 1], frame[1, 1], frame[0, 2],
                                             frame[1, 2]])
    np.testing.assert_array_equal(bm[:, 1], [frame[2, 0], frame[3, 0], frame[2, 1], frame[3, 1], frame[2, 2],
                                             frame[3, 2]])


def test_bidirectional_reverses_even_lines():
    # 2 lines x 3 pixels, bidirectional, 2 knots: the second line is scanned right to left
    tmpl = np.zeros((2, 3))
    s = prep.init_settings({"nknots": 2, "isbidirectional": True}, tmpl, 2, 3)
    dwell = 1 / 6
    t = dwell / 2 + np.array([[0, 1, 2], [5, 4, 3]]) / 6
    np.testing.assert_allclose(s["tfrac"], t, rtol=0, atol=1e-15)  # one knot interval [0, 1]
    lay = prep.block_layout(s)
    np.testing.assert_allclose(lay.tfrac[:, 0], [t[0, 0], t[1, 0], t[0, 1], t[1, 1], t[0, 2], t[1, 2]], atol=1e-15)


def test_non_integer_lines_per_knot():
    # 5 lines x 2 pixels, 3 knots: 2.5 lines per knot, knot times linspace(0, 1, 3) over the data;
    # scan time 1/20 + (2 l + j) / 10, so pixels (0,0) (0,1) (1,0) (1,1) (2,0) fall before t = 1/2
    tmpl = np.zeros((5, 2))
    s = prep.init_settings({"nknots": 3}, tmpl, 5, 2)
    np.testing.assert_allclose(s["t_knots"], [0, 0.5, 1], atol=1e-15)
    np.testing.assert_array_equal(s["prevknotind"], [[1, 1], [1, 1], [1, 2], [2, 2], [2, 2]])
    lay = prep.block_layout(s)
    assert (lay.frame_h, lay.frame_w) == (5, 2)
    # block 1 in column-major order: (0,0) (1,0) (2,0) (0,1) (1,1); tfrac = t / (1/2)
    np.testing.assert_allclose(lay.tfrac[:, 0], [0.1, 0.5, 0.9, 0.3, 0.7], rtol=0, atol=1e-15)
    # block 2: (3,0) (4,0) (2,1) (3,1) (4,1); tfrac = (t - 1/2) / (1/2)
    np.testing.assert_allclose(lay.tfrac[:, 1], [0.3, 0.7, 0.1, 0.5, 0.9], rtol=0, atol=1e-15)
    np.testing.assert_array_equal(lay.min_points, [1, 1, 0])


def test_cropping_removes_rows_and_columns():
    # cropping [left right bottom top] = [1 0 1 0] on 5 lines x 4 pixels: the data keeps lines 1..4
    # and pixels 1..3 (0-based); with a template of the cropped size, subrec = [0 3 0 4]
    tmpl = np.zeros((4, 3))
    s = prep.init_settings({"nknots": 3, "cropping": [1, 0, 1, 0], "basex": np.zeros((4, 3)),
                            "basey": np.zeros((4, 3))}, tmpl, 5, 4)
    assert s["subrec"] == [0, 3, 0, 4]  # [1 - left, tw + right, 1 - bottom, th + top]
    dwell = 1 / 20
    pst = dwell / 2 + np.arange(20).reshape(5, 4) / 20
    crop = pst[1:, 1:]
    # integer lines per knot on the cropped data (4 / 2): knotlines = 1:2:4 index the UNCROPPED scan
    # times (steady_scan.m:795-797), i.e. full-frame lines 0 and 2, so the second knot time is the
    # start of full line 2 (0.4) and only cropped line 0 (full line 1) falls before it
    tk = [0.0, pst[2, :].min() - dwell / 2, 1.0]
    np.testing.assert_allclose(s["t_knots"], tk, atol=1e-15)
    np.testing.assert_allclose(tk[1], 0.4, atol=1e-15)
    np.testing.assert_array_equal(s["prevknotind"], [[1, 1, 1], [2, 2, 2], [2, 2, 2], [2, 2, 2]])
    np.testing.assert_array_equal(s["prevknotind"], np.where(crop < tk[1], 1, 2))


def test_template_gradients_nan_padded():
    t = np.array([[1.0, 2.0, 4.0], [3.0, 7.0, 11.0]])
    xg, yg = prep.template_gradients(t)
    np.testing.assert_array_equal(xg[:, :2], [[1, 2], [4, 4]])
    assert np.isnan(xg[:, 2]).all()
    np.testing.assert_array_equal(yg[0], [2, 5, 7])
    assert np.isnan(yg[1]).all()
