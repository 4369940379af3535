"""Parity with the FP64 oracle at the frame shapes the benchmarks run (through the C ABI).

Each case takes a few frames of one measured shape, so the oracle finishes in seconds:

* 512x512, knots every 2 lines (257 knots, Hb = 1024, W = 256), the single-session throughput shape;
* 256x256, knots every 4 lines, lambda 1e-2, at most 30 iterations, the plain-method small shape;
* 796x512 and 128x128 (lines x pixels), knots every line, lambda 1e-2, move threshold 1e-3 px, at
  most 30 iterations, two shapes of the ragged batch;
* 512x512 with frames whose vertical offsets differ by ~38 px inside one tile of frames, so the
  template rows a tile needs do not fit its shared-memory window and precision S samples the
  global template instead (the fallback path of the trial rounds and the assembly).

Precision D must reproduce the oracle's iterations, stop reason and masks exactly and its knots to
1e-6 px. Precision S (FP32 pixel arithmetic, FP64 reduction and solve) is held to 0.02 px RMS on
the frames the reference's caller accepts (steady_scan.m:246-284: a frame with no block inside the
template, or with a correlation below corr_thresh, is marked failed and its knots are not used).
"""
import os

import numpy as np
import pytest

from oracle import oracle
from steadyscan_b200 import api, prep, synth
from tests.helpers import make_args

pytestmark = pytest.mark.gpu

KNOT_TOL_D = 1e-6   # px, precision D
KNOT_RMS_S = 0.02   # px RMS, precision S
THREADS = os.cpu_count() or 1

SHAPES = {
    "512x512_k2": dict(nlines=512, linewidth=512, nknots=257, n_frames=4, seed=201, n_blobs=400, sigma=(2.0, 6.0),
                       walk_sigma=0.1, clip_px=10.0, jumps=(0, 3), jump_px=4.0, frame_dtype=np.uint16,
                       settings={"lambda": 5e-3}),
    "256x256_k4": dict(nlines=256, linewidth=256, nknots=65, n_frames=8, seed=202, n_blobs=80, sigma=(2.0, 5.0),
                       walk_sigma=0.15, clip_px=6.0, jumps=1, jump_px=4.0, frame_dtype=np.uint16,
                       settings={"lambda": 1e-2, "max_iter": 30}),
    "796x512_k1": dict(nlines=796, linewidth=512, nknots=797, n_frames=4, seed=203, n_blobs=497, sigma=(2.0, 5.0),
                       walk_sigma=0.15, clip_px=6.0, jumps=1, jump_px=4.0, frame_dtype=np.uint16,
                       settings={"lambda": 1e-2, "max_iter": 30, "move_thresh": 1e-3}),
    "128x128_k1": dict(nlines=128, linewidth=128, nknots=129, n_frames=8, seed=204, n_blobs=20, sigma=(2.0, 5.0),
                       walk_sigma=0.15, clip_px=6.0, jumps=1, jump_px=4.0, frame_dtype=np.uint16,
                       settings={"lambda": 1e-2, "max_iter": 30, "move_thresh": 1e-3}),
}

_CACHE = {}


def _case(name):
    if name not in _CACHE:
        args, rec, s = make_args(**SHAPES[name])
        _CACHE[name] = (args, oracle.align_group(args, n_threads=THREADS), s)
    return _CACHE[name]


def accepted_frames(o, args, settings):
    """Frames the reference's caller keeps (steady_scan.m:246-284): some block inside the template
    and a correlation of at least corr_thresh."""
    w = args["tfrac"].shape[1]
    n = int(args["nFrames"])
    used = o["mask"].reshape(o["mask"].shape[0], n, w).any(axis=0)   # [frame, block]
    corr = np.asarray(o["frame_corr"])
    return used.any(axis=1) & (corr >= settings["corr_thresh"])


def knots_rms(g, o, args, frames):
    w1 = args["tfrac"].shape[1] + 1
    n = int(args["nFrames"])
    sel = np.repeat(frames, w1)
    d = np.concatenate([(g["dx"] - o["dx"])[sel], (g["dy"] - o["dy"])[sel]])
    return float(np.sqrt(np.mean(d * d))) if d.size else 0.0


@pytest.mark.parametrize("name", list(SHAPES))
def test_precision_d_matches_oracle_at_benchmark_shapes(name):
    args, o, _ = _case(name)
    g = api.align_group(args)
    assert g["iter_used"] == o["iterations"], (g["iter_used"], o["iterations"])
    assert g["stop_reason"] == o["stop_reason"]
    np.testing.assert_allclose(g["dx"], o["dx"], atol=KNOT_TOL_D, rtol=0)
    np.testing.assert_allclose(g["dy"], o["dy"], atol=KNOT_TOL_D, rtol=0)
    np.testing.assert_array_equal(g["mask"], o["mask"])
    np.testing.assert_allclose(g["frame_corr"], o["frame_corr"], atol=1e-9, rtol=1e-9, equal_nan=True)
    np.testing.assert_allclose(g["residrms"], o["residrms"], atol=1e-9, rtol=1e-9, equal_nan=True)


def fp64_spread(args, o, frames, rel=1e-7, seed=0):
    """RMS change of the FP64 oracle's knots when the template (and its gradients) is perturbed by
    ``rel`` relative noise, the rounding of FP32 template storage: how far the reference algorithm
    itself moves under input changes of the size that FP32 pixel arithmetic makes."""
    rng = np.random.default_rng(seed)
    t = np.asarray(args["template_image"]) * (1 + rel * rng.standard_normal(np.shape(args["template_image"])))
    a = dict(args, template_image=t)
    a["xgrad"], a["ygrad"] = prep.template_gradients(t)
    p = oracle.align_group(a, n_threads=THREADS)
    return knots_rms(p, o, args, frames)


# Shapes whose estimate the FP64 algorithm itself does not pin down: with a knot every line on
# 128-pixel lines, many blocks cross little template structure and the solution wanders (the FP64
# oracle's knots move ~1 px RMS, tens of px at worst, under a 1e-7 relative template change). There
# precision S is held to the FP64 path's own spread instead of the fixed bound.
ILL_CONDITIONED = {"128x128_k1"}


@pytest.mark.parametrize("name", list(SHAPES))
def test_precision_s_within_bound_at_benchmark_shapes(name):
    args, o, s = _case(name)
    g = api.align_group(dict(args, flags="S"))
    keep = accepted_frames(o, args, s)
    assert keep.any()
    rms = knots_rms(g, o, args, keep)
    if name in ILL_CONDITIONED:
        spread = fp64_spread(args, o, keep)
        assert spread > KNOT_RMS_S, spread  # the shape is as ill-conditioned as stated
        assert rms <= max(KNOT_RMS_S, spread), (rms, spread)
    else:
        assert rms <= KNOT_RMS_S, (rms, keep)
        # the well-conditioned shapes barely move under the same perturbation
        assert fp64_spread(args, o, keep) <= 1e-3
    # valid-pixel counts differ at most at boundary ties
    assert abs(int(g["mask"].sum()) - int(o["mask"].sum())) <= 0.001 * g["mask"].size


def _offset_frames_args(seed=211, n_frames=4):
    """512x512 frames, knots every 2 lines, whose vertical offset ramps from -32 to +32 px over the
    frames (at one block column the frames of a tile lie ~38 px apart: more template rows than an
    assembly or trial window holds), started from the true knots plus 0.3 px of noise."""
    rng = np.random.default_rng(seed)
    h = w = 512
    nk = 257
    tmpl = synth.make_template(h, w, 400, (2.0, 6.0), rng)
    walk = synth.make_walk(h * (n_frames + 1), 0.1, 3.0, (0, 1), h, 2.0, rng)
    walk[:, 1] += np.linspace(-32.0, 32.0, walk.shape[0])
    frames = synth.render_frames(tmpl, walk[:h * n_frames], h, w, rng)
    s = prep.init_settings({"nknots": nk, "lambda": 5e-3}, tmpl, h, w)
    lay = prep.block_layout(s)
    bm = prep.frames_to_blockmatrix(np.clip(np.rint(frames), 0, 65535).astype(np.uint16), lay, dtype=np.uint16)
    tx, ty = synth.truth_knots(walk, h, nk, n_frames)
    ex = tx + rng.normal(0, 0.3, tx.shape)
    ey = ty + rng.normal(0, 0.3, ty.shape)
    return prep.boundary_arguments(s, tmpl, bm, n_frames, ex, ey, layout=lay), s


def test_precision_s_global_template_path_at_512():
    args, s = _offset_frames_args()
    o = oracle.align_group(args, n_threads=THREADS)
    gd = api.align_group(args)
    np.testing.assert_allclose(gd["dx"], o["dx"], atol=KNOT_TOL_D, rtol=0)
    np.testing.assert_allclose(gd["dy"], o["dy"], atol=KNOT_TOL_D, rtol=0)
    assert gd["iter_used"] == o["iterations"]
    b = api.Batch([dict(args, flags="S")], want_mask=True)
    b.run()
    g = b.collect()[0]
    st = b.stats()["staging"]
    b.close()
    # the tiles of these frames did not fit the window: some trial tiles and some assembly tiles
    # sampled the global template
    assert st["ls_windowed"] < st["ls_ctas"], st
    assert st["eval_windowed"] < st["eval_ctas"], st
    keep = accepted_frames(o, args, s)
    assert keep.any()
    assert knots_rms(g, o, args, keep) <= KNOT_RMS_S
