"""The tile schedule (frames per evaluation tile) changes no precision-D result and precision-S
results only at FP32 rounding level (tiles of at least 4 frames read the template from a shared-
memory window, smaller ones from global memory, with a different rounding of the bilinear sample);
the autotuner picks one of its candidates per group shape and caches it."""
import json

import numpy as np
import pytest

from steadyscan_b200 import api
from steadyscan_b200.autotune import Autotuner, shape_key
from tests.helpers import make_args

pytestmark = pytest.mark.gpu


def _groups():
    out = []
    for i, s in enumerate([dict(nlines=64, linewidth=64, nknots=33, n_frames=40, seed=90, n_blobs=30),
                           dict(nlines=64, linewidth=64, nknots=33, n_frames=7, seed=91, n_blobs=30),
                           dict(nlines=32, linewidth=48, nknots=9, n_frames=20, seed=92, n_blobs=20)]):
        a = make_args(frame_dtype=np.uint16, **s)[0]
        a["flags"] = "S"
        out.append(a)
    return out


@pytest.mark.parametrize("flags", ["S", "D"])
def test_frames_per_tile_changes_no_result(flags):
    groups = [dict(g, flags=flags) for g in _groups()]
    ref = api.align_groups(groups)
    for fpc in (1, 3, 8, 64):
        got = api.align_groups([dict(g, frames_per_cta=fpc) for g in groups])
        for a, b in zip(ref, got):
            if flags == "D":
                assert a["iter_used"] == b["iter_used"]
                np.testing.assert_array_equal(a["dx"], b["dx"])
                np.testing.assert_array_equal(a["dy"], b["dy"])
                np.testing.assert_array_equal(a["mask"], b["mask"])
            else:
                d = np.concatenate([a["dx"] - b["dx"], a["dy"] - b["dy"]])
                assert np.sqrt(np.mean(d * d)) <= 1e-3 and np.abs(d).max() <= 1e-2


def test_frames_per_tile_out_of_range_is_an_error():
    g = _groups()[0]
    with pytest.raises(api.SteadyScanError):
        api.align_group(dict(g, frames_per_cta=65))


def test_autotuner_picks_a_candidate_per_shape_and_caches(tmp_path):
    groups = _groups()
    path = str(tmp_path / "tune.json")
    t = Autotuner(cache_path=path, reps=1)
    tuned = t.apply(groups)
    keys = {shape_key(g) for g in groups}
    assert set(t.choices) == keys
    for g, tg in zip(groups, tuned):
        assert tg["frames_per_cta"] == t.choices[shape_key(g)]
        assert tg["frames_per_cta"] in t.timings[shape_key(g)]
    with open(path) as f:
        assert any(set(v) == keys for v in json.load(f).values())
    # a second tuner reads the cache and times nothing
    t2 = Autotuner(cache_path=path)
    t2.apply(groups)
    assert t2.timings == {} and t2.choices == t.choices
    for a, b in zip(api.align_groups(groups), api.align_groups(tuned)):
        np.testing.assert_allclose(a["dx"], b["dx"], atol=1e-2, rtol=0)
    # validation on the whole batch keeps the faster of the tuned and the default split
    v = t2.apply(groups, validate=True)
    lv = t2.last_validation
    assert lv is not None and lv["kept"] in ("tuned", "default")
    want = [0] * len(groups) if lv["kept"] == "default" else [t.choices[shape_key(g)] for g in groups]
    assert [g["frames_per_cta"] for g in v] == want
