"""ss_prepare_frames on the GPU against the oracle's restatement of the reference driver's frame
preparation (prefilter_foralignment, cropimage, image2blockmatrix; steady_scan.m:229-234, 625-643,
830-834): block matrices exactly, the FFT blur and median normalisation to FP64 rounding."""
import types

import numpy as np
import pytest

from oracle import frontend
from steadyscan_b200 import api, prep
from tests.helpers import make_args

pytestmark = pytest.mark.gpu


def _case(n_frames=3, seed=4, **kw):
    args, _, s = make_args(n_frames=n_frames, seed=seed, **kw)
    lay = prep.block_layout(s)
    crop = lay.cropping if lay.cropping else [0, 0, 0, 0]
    h = lay.prevknotind.shape[0] + crop[2] + crop[3]
    w = lay.prevknotind.shape[1] + crop[0] + crop[1]
    rng = np.random.default_rng(seed)
    frames = rng.integers(0, 60000, size=(h, w, n_frames)).astype(np.uint16)
    return args, lay, frames


def _device(frames):
    import torch
    return torch.from_numpy(np.ascontiguousarray(frames.transpose(2, 1, 0))).cuda().permute(2, 1, 0)


@pytest.mark.parametrize("kw", [dict(), dict(settings={"cropping": [2, 3, 0, 0]}),
                                dict(settings={"isbidirectional": True}), dict(nlines=30, linewidth=20, nknots=8)])
def test_block_matrix_exact(kw):
    _, lay, frames = _case(**kw)
    ref = frontend.set_bmdata(frames, lay.prevknotind, lay.frame_w, lay.cropping, 0.0, False)
    for src in (frames, _device(frames)):
        u16 = api.prepare_frames(src, lay, out_dtype=np.uint16).cpu().numpy().astype(np.float64)
        f64 = api.prepare_frames(src, lay, out_dtype=np.float64).cpu().numpy()
        np.testing.assert_array_equal(u16, ref)
        np.testing.assert_array_equal(f64, ref)


@pytest.mark.parametrize("gsd,mednorm", [(1.5, False), (0.8, True), (0.0, True), (3.2, True)])
def test_prefilter_matches_fft(gsd, mednorm):
    _, lay, frames = _case(n_frames=4, seed=9)
    ref = frontend.set_bmdata(frames, lay.prevknotind, lay.frame_w, lay.cropping, gsd, mednorm)
    for src in (frames, _device(frames)):
        got = api.prepare_frames(src, lay, pregauss=gsd, mednorm=mednorm).cpu().numpy()
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


def test_vertical_cropping_with_a_synthetic_block_map():
    rng = np.random.default_rng(3)
    h, w, n, crop = 40, 30, 2, [2, 3, 4, 1]
    hc, wc = h - crop[2] - crop[3], w - crop[0] - crop[1]
    blockind = rng.integers(1, 8, size=(hc, wc))
    lay = types.SimpleNamespace(prevknotind=blockind, frame_w=7, cropping=crop)
    frames = rng.uniform(0, 100, size=(h, w, n)).astype(np.float32)
    ref = frontend.set_bmdata(frames, blockind, 7, crop, 1.1, True)
    got = api.prepare_frames(frames, lay, pregauss=1.1, mednorm=True).cpu().numpy()
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    ref0 = frontend.set_bmdata(frames, blockind, 7, crop, 0.0, False)
    got0 = api.prepare_frames(frames, lay, out_dtype=np.float32).cpu().numpy()
    np.testing.assert_array_equal(got0, ref0.astype(np.float32))


def test_device_prepared_frames_align_like_the_host_path():
    """The recording's uint16 frames block-reordered on the device align exactly as the same frames
    block-reordered on the host (make_args' bmData)."""
    args, rec, s = make_args(n_frames=4, seed=21, frame_dtype=np.uint16)
    lay = prep.block_layout(s)
    dev = api.prepare_frames(_device(rec.frames_as(np.uint16)), lay, out_dtype=np.uint16)
    np.testing.assert_array_equal(dev.cpu().numpy(), np.asarray(args["bmData"]))
    g0 = api.align_group(dict(args, flags="D"))
    g1 = api.align_group(dict(args, bmData=dev, flags="D"))
    assert g0["iter_used"] == g1["iter_used"]
    np.testing.assert_array_equal(g0["dx"], g1["dx"])
    np.testing.assert_array_equal(g0["dy"], g1["dy"])
