"""The corrected-frame helper used by the accuracy reports (CPU)."""
import numpy as np

from steadyscan_b200 import correct, synth
from tests.helpers import make_args


def test_truth_knots_correct_frames_onto_the_template():
    args, rec, s = make_args(nlines=32, linewidth=32, nknots=9, n_frames=3, seed=5, noise=False, clip_px=2.0)
    n = 3
    tdx, tdy = synth.truth_knots(rec.walk, 32, 9, n)
    ht, wt = rec.template.shape
    corr_t, w_t = correct.correct_frames(args["bmData"], tdx.T.reshape(-1), tdy.T.reshape(-1), args["tfrac"],
                                         args["basex"], args["basey"], args["base_mask"], n, (ht, wt))
    zero = np.zeros(9 * n)
    corr_0, w_0 = correct.correct_frames(args["bmData"], zero, zero, args["tfrac"], args["basex"], args["basey"],
                                         args["base_mask"], n, (ht, wt))
    tmpl = np.broadcast_to(rec.template, corr_t.shape)
    ones = np.ones_like(corr_t)
    err_truth = correct.relative_l2(corr_t, w_t, tmpl, ones)
    err_zero = correct.relative_l2(corr_0, w_0, tmpl, ones)
    assert err_truth < 0.1
    assert err_truth < 0.5 * err_zero


def test_relative_l2_of_identical_corrections_is_zero():
    a = np.random.default_rng(0).random((2, 5, 5))
    w = np.ones_like(a)
    assert correct.relative_l2(a, w, a, w) == 0.0
