"""The FP64 oracle against whole align_group_to_template runs of the reference's own task layer
(Task::alignFrames, MainIteration::execute, its kernels, filters and solver id 1, host-compiled
from the reference tree; tests/golden/make_refrun_golden.py): the Gauss-Newton trajectory, the line
search, the iteration control and the stop criteria, pinned iteration by iteration."""
import glob
import os

import numpy as np
import pytest

from oracle import oracle

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "refrun_*.npz")))


def _args(z):
    a = {k[3:]: z[k] for k in z.files if k.startswith("in_")}
    a["flags"] = str(a["flags"])
    for k in ("group_size", "nFrames", "max_iter", "max_filter_iterations", "solver_id", "filter_id",
              "gpu_device_id"):
        a[k] = int(a[k])
    return a


@pytest.fixture(scope="module", autouse=True)
def _build():
    oracle.build()


def test_fixtures_present():
    assert len(GOLDEN) >= 16
    assert sum("t" in str(np.load(p)["in_flags"]) for p in GOLDEN) >= 3  # TimedMainIteration runs


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p)[7:-4] for p in GOLDEN])
def test_trajectory_matches_reference_run(path):
    z = np.load(path)
    o = oracle.align_group(_args(z), want_history=True)
    it = int(z["iterations"])
    assert o["iterations"] == it
    assert o["stop_reason"] == int(z["stop_reason"])
    np.testing.assert_array_equal(o["mask"], z["mask"])
    # the knot chain after every iteration, the final per-frame knots and the iteration control's
    # correlations (the restatement contracts a*b+c into fma like nvcc; the host build does not)
    np.testing.assert_allclose(o["all_params"][:it], z["all_params"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(o["dx"], z["dx"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(o["dy"], z["dy"], rtol=0, atol=1e-9)
    np.testing.assert_allclose(o["iter_corr"][:it], z["iter_corr"], rtol=1e-10, atol=1e-12)
    # errvals are saved only for iterations that go on to the next one (task.cpp:362-372): the
    # same entries are written (NaN in the fixture marks an unwritten one, zero in the oracle's)
    written = ~np.isnan(z["iter_errvals"])
    assert not np.any(o["iter_errvals"][:2 * it][~written])
    np.testing.assert_allclose(o["iter_errvals"][:2 * it][written], z["iter_errvals"][written], rtol=1e-10, atol=1e-9)
    np.testing.assert_allclose(o["frame_corr_hist"][:it], z["frame_corr_hist"], rtol=1e-10, atol=1e-12)
    np.testing.assert_allclose(o["frame_corr"], z["frame_corr"], rtol=1e-10, atol=1e-12, equal_nan=True)
    np.testing.assert_allclose(o["residrms"], z["residrms"], rtol=1e-10, atol=1e-12, equal_nan=True)
    if "rg_params" in z.files:  # flag t: the chain after every half-step; later slots stay zero
        k = z["rg_params"].shape[0]
        np.testing.assert_allclose(o["rg_params"][:k], z["rg_params"], rtol=0, atol=1e-9)
        assert not np.any(o["rg_params"][k:])
