"""Frame preparation (prefilter_foralignment, cropimage, image2blockmatrix; steady_scan.m:229-234,
625-643, 830-834) on the CPU: the oracle's FFT blur against the direct circular convolution that the
GPU kernels evaluate, the oracle's block reorder against the library's host path and hand-made
cases, and argument checks of ss_prepare_frames before any device work."""
import ctypes as C
import math

import numpy as np
import pytest

from oracle import frontend
from steadyscan_b200 import _lib, build, prep
from tests.helpers import make_args


def _direct_blur(img, gsd):
    """Two 1-D circular passes with the taps within ceil(9.6 gsd) of the centre, each axis
    normalised by its sum over the padded period (the formulation of ss_frontend.cuh)."""
    h, w = img.shape
    L = math.ceil(math.sqrt((2 * gsd ** 2) * math.log(10000 / (math.sqrt(2 * math.pi) * gsd))))

    def taps(period):
        d = np.arange(period)
        g = np.exp(-np.minimum(d, period - d) ** 2 / (2 * gsd ** 2))
        R = min(math.ceil(9.6 * gsd), (period - 1) // 2)
        return g[:R + 1] / g.sum(), R

    def circ(x, axis, period):
        t, R = taps(period)
        n = x.shape[axis]
        out = np.zeros_like(x)
        for i in range(n):
            acc = 0.0
            for d in range(-R, R + 1):
                a = (i + d) % period
                if a < n:
                    acc = acc + (x[a, :] if axis == 0 else x[:, a]) * t[abs(d)]
            if axis == 0:
                out[i, :] = acc
            else:
                out[:, i] = acc
        return out

    return circ(circ(img, 0, h + L), 1, w + L)


@pytest.mark.parametrize("gsd", [0.7, 1.5, 3.0])
def test_fft_blur_equals_direct_circular_taps(gsd):
    rng = np.random.default_rng(int(gsd * 10))
    img = rng.uniform(0, 1000, size=(37, 29))
    fft = frontend.prefilter_foralignment(img, gsd, False)[:, :, 0]
    direct = _direct_blur(img, gsd)
    np.testing.assert_allclose(direct, fft, rtol=0, atol=1e-11 * np.abs(fft).max())


def test_median_normalisation_divides_each_frame_by_its_median():
    rng = np.random.default_rng(2)
    d = rng.uniform(1, 9, size=(6, 5, 3))
    out = frontend.prefilter_foralignment(d, 0, True)
    for k in range(3):
        np.testing.assert_allclose(out[:, :, k], d[:, :, k] / np.median(d[:, :, k]), rtol=1e-15)


def test_image2blockmatrix_hand_made():
    # a 3 x 2 image, blocks numbered column-major 1 2 1 / 2 2 1: block 1 = x(1,1), x(3,1), x(3,2)
    x = np.array([[1, 4], [2, 5], [3, 6]], dtype=np.float64)
    bi = np.array([[1, 2], [2, 2], [1, 1]])
    y = frontend.image2blockmatrix(x, bi, 2)
    np.testing.assert_array_equal(y, np.array([[1, 2], [3, 4], [6, 5]], dtype=np.float64))


@pytest.mark.parametrize("case", ["plain", "cropped", "bidirectional", "nonint"])
def test_host_blockmatrix_matches_oracle(case):
    kw = {"plain": dict(), "cropped": dict(settings={"cropping": [2, 3, 0, 0]}),
          "bidirectional": dict(settings={"isbidirectional": True}), "nonint": dict(nlines=30, linewidth=20, nknots=8)}[case]
    args, _, s = make_args(n_frames=3, seed=4, **kw)
    lay = prep.block_layout(s)
    rng = np.random.default_rng(5)
    crop = lay.cropping if lay.cropping else [0, 0, 0, 0]
    h = lay.prevknotind.shape[0] + crop[2] + crop[3]
    w = lay.prevknotind.shape[1] + crop[0] + crop[1]
    frames = rng.integers(0, 60000, size=(h, w, 3)).astype(np.uint16)
    host = prep.frames_to_blockmatrix(frames, lay, dtype=np.float64)
    ref = frontend.set_bmdata(frames, lay.prevknotind, lay.frame_w, lay.cropping, 0.0, False)
    np.testing.assert_array_equal(host, ref)


def test_prepare_frames_rejects_bad_arguments_before_device_work():
    build.build()
    lib = _lib.load()
    frames = np.zeros((8, 6 * 2), np.uint16, order="F")
    gather = np.full((4, 3), -1, np.int32, order="F")
    out = _lib.SSMatrix(None, 4, 6, _lib.SS_F64, _lib.SS_DEVICE)

    def call(crop, g=gather, o=out):
        p = _lib.SSPrepFrames(_lib.SSMatrix(frames.ctypes.data, 8, 12, _lib.SS_U16, _lib.SS_HOST), 2, 0.0, 0,
                              (C.c_int32 * 4)(*crop), g.ctypes.data, g.shape[0], g.shape[1], o, 0)
        return lib.ss_prepare_frames(C.byref(p))

    assert call([3, 3, 0, 0]) == -1  # cropping removes every column
    bad = gather.copy(order="F")
    bad[0, 0] = 48  # outside the 8 x 6 frame
    assert call([0, 0, 0, 0], g=bad) == -1
    assert call([0, 0, 0, 0]) == -1  # out has no device buffer
