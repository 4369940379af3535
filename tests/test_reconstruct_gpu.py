"""ss_reconstruct_frames (invert_bilinear_sampling, steady_scan.m:290-404) against the oracle's
restatement. The iteration's stopping rule compares FP32 energies whose linear term the reference
sums in its BLAS's order; near convergence the decrease per check is an ulp, so the sweep counts of
two summation orders differ. The arithmetic is therefore checked by replaying the GPU's sweep counts
in the oracle (iterates to FP32 rounding), and the stopping rule separately (counts within a few
check intervals, outputs close where the iterates have converged)."""
import numpy as np
import pytest

from oracle import oracle
from oracle import reconstruct as rc
from steadyscan_b200 import api, prep, synth
from tests.helpers import make_args

pytestmark = pytest.mark.gpu


def _estimated(seed, n_frames=6, **kw):
    args, rec, s = make_args(n_frames=n_frames, seed=seed, **kw)
    o = oracle.align_group(dict(args, flags="D"))
    nk = args["tfrac"].shape[1] + 1
    dxk = np.asarray(o["dx"]).reshape(nk, -1, order="F")
    dyk = np.asarray(o["dy"]).reshape(nk, -1, order="F")
    return rec, s, dxk, dyk


def _subpixel():
    from scipy.ndimage import map_coordinates
    rng = np.random.default_rng(1)
    n = 24
    tmpl = synth.make_template(n, n, 6, (2.0, 3.0), rng)
    s = prep.init_settings({"nknots": 5, "ibs_regfac": 1e-4}, tmpl, n, n)
    frame = map_coordinates(tmpl, [s["basey"] - 1 + 0.21, s["basex"] - 1 + 0.37], order=1, mode="nearest")
    fr = np.stack([frame] * 3, 2).astype(np.float32)
    return tmpl, s, fr, np.full((5, 3), 0.37), np.full((5, 3), 0.21)


def _oracle(fr, dxk, dyk, s, shape, stop_at=None):
    return rc.invert_bilinear_sampling(fr, dxk, dyk, s["basex"], s["basey"], s["tfrac"], s["prevknotind"], *shape,
                                       regfac=s.get("ibs_regfac", 3e-3),
                                       aspect=s.get("ibs_template_pixel_aspect_ratio", 1.0), stop_at=stop_at)


@pytest.mark.parametrize("seed", [5, 7, 11])
def test_iterates_match_the_oracle_at_the_same_sweeps(seed):
    rec, s, dxk, dyk = _estimated(seed)
    fr = rec.frames.astype(np.float32)
    shape = rec.template.shape
    g = api.reconstruct_frames(fr, dxk, dyk, s, shape)
    o_out, o_mask, o_its = _oracle(fr, dxk, dyk, s, shape, stop_at=list(g["iterations"]))
    np.testing.assert_array_equal(g["mask"], o_mask)
    assert o_its == list(g["iterations"])
    m = o_mask
    scale = np.abs(o_out[m]).max()
    np.testing.assert_allclose(g["data_corrected"][m], o_out[m], rtol=0, atol=1e-4 * scale)
    assert np.all(np.isnan(g["data_corrected"][~m]))


def test_stopping_rule_close_to_the_oracle():
    rec, s, dxk, dyk = _estimated(5)
    fr = rec.frames.astype(np.float32)
    g = api.reconstruct_frames(fr, dxk, dyk, s, rec.template.shape)
    o_out, o_mask, o_its = _oracle(fr, dxk, dyk, s, rec.template.shape)
    its = np.array(g["iterations"])
    assert np.all(np.abs(its - np.array(o_its)) <= 10 * 2), (its, o_its)  # within two of the largest interval
    m = o_mask
    d = np.abs(g["data_corrected"][m] - o_out[m])
    assert np.median(d) < 1e-3 * np.abs(o_out[m]).max()


def test_subpixel_frames_reconstruct_the_template_and_device_frames_equal_host():
    import torch
    tmpl, s, fr, dx, dy = _subpixel()
    g = api.reconstruct_frames(fr, dx, dy, s, tmpl.shape)
    dev = torch.from_numpy(np.ascontiguousarray(fr.transpose(2, 1, 0))).cuda().permute(2, 1, 0)
    gd = api.reconstruct_frames(dev, dx, dy, s, tmpl.shape, out_dtype=np.float64)
    np.testing.assert_array_equal(np.nan_to_num(g["data_corrected"]), np.nan_to_num(gd["data_corrected"]).astype(np.float32))
    for k in range(3):
        m = g["mask"][:, :, k]
        assert m.sum() > 0.9 * m.size
        assert np.median(np.abs(g["data_corrected"][:, :, k][m] - tmpl[m])) < 1e-2 * tmpl.max()


def test_extra_channel_uses_the_same_knots():
    """An extra channel (steady_scan.m:137-154) is the same reconstruction of the channel's frames
    with the knots estimated on the main channel."""
    rec, s, dxk, dyk = _estimated(7, n_frames=4)
    extra = (0.5 * rec.frames + 20.0).astype(np.float32)
    g = api.reconstruct_frames(extra, dxk, dyk, s, rec.template.shape)
    o_out, o_mask, _ = _oracle(extra, dxk, dyk, s, rec.template.shape, stop_at=list(g["iterations"]))
    np.testing.assert_array_equal(g["mask"], o_mask)
    m = o_mask
    np.testing.assert_allclose(g["data_corrected"][m], o_out[m], rtol=0, atol=1e-4 * np.abs(o_out[m]).max())


def test_frames_that_constrain_nothing_are_skipped():
    rec, s, dxk, dyk = _estimated(5, n_frames=4)
    dxk = dxk.copy()
    dxk[:, 1] += 1000.0  # frame 1 maps entirely off the template
    fr = rec.frames.astype(np.float32)
    g = api.reconstruct_frames(fr, dxk, dyk, s, rec.template.shape)
    assert g["iterations"][1] == 0
    assert not g["mask"][:, :, 1].any() and np.all(np.isnan(g["data_corrected"][:, :, 1]))
    o_out, o_mask, o_its = _oracle(fr, dxk, dyk, s, rec.template.shape, stop_at=list(g["iterations"]))
    assert o_its[1] == 0
    m = o_mask
    np.testing.assert_allclose(g["data_corrected"][m], o_out[m], rtol=0, atol=1e-4 * np.abs(o_out[m]).max())
