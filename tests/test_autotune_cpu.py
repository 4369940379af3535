"""Host logic of the autotuner: shape keys, probe selection and the choice cache (no GPU)."""
import json

import numpy as np

from steadyscan_b200 import autotune


def _group(hb, w, nf, flags="S", tshape=(40, 40)):
    return {"tfrac": np.zeros((hb, w)), "nFrames": nf, "flags": flags, "template_image": np.zeros(tshape),
            "bmData": np.zeros((hb, w * nf), dtype=np.uint16)}


def test_shape_key_separates_shapes_precisions_and_storage():
    a, b = _group(64, 8, 4), _group(64, 16, 4)
    assert autotune.shape_key(a) != autotune.shape_key(b)
    assert autotune.shape_key(a) != autotune.shape_key(dict(a, flags="D"))
    assert autotune.shape_key(a) != autotune.shape_key(a, template_storage="f16")
    assert autotune.shape_key(a) == autotune.shape_key(dict(a, nFrames=9))  # length is not part of the key
    # gradients that are the template's forward differences sample the template window; others not
    t = np.arange(1600.0).reshape(40, 40) % 7
    xg = np.hstack([np.diff(t, axis=1), np.full((40, 1), np.nan)])
    yg = np.vstack([np.diff(t, axis=0), np.full((1, 40), np.nan)])
    derived = dict(a, template_image=t, xgrad=xg, ygrad=yg)
    assert autotune.shape_key(derived) == autotune.shape_key(dict(a, template_image=t))
    assert autotune.shape_key(derived) != autotune.shape_key(dict(derived, xgrad=2 * xg))


def test_probe_takes_the_largest_groups_and_fills_the_gpu():
    t = autotune.Autotuner(probe_groups=2, probe_frames=100, min_tiles=1000, max_repeat=16)
    gs = [_group(64, 10, n) for n in (5, 60, 30, 50)]
    p = t._probe(gs)
    base = [g["nFrames"] for g in p[:2]]
    assert base == [60, 30]  # largest first; 50 would exceed probe_frames after 60
    tiles = 10 * 2 + 10 * 1  # block columns x chunks of at most 32 frames
    assert len(p) == 2 * min(16, -(-1000 // tiles))


def test_choices_are_cached_per_device(tmp_path):
    path = str(tmp_path / "c.json")
    t = autotune.Autotuner(cache_path=path)
    t.choices = {"k1": 16}
    t._save()
    data = json.load(open(path))
    assert data[t._device] == {"k1": 16}
    t2 = autotune.Autotuner(cache_path=path)
    assert t2.choices == {"k1": 16}
    # a tuned key is not timed again (tune() would need a GPU otherwise)
    g = _group(64, 8, 4)
    t2.choices[autotune.shape_key(g)] = 8
    assert t2.tune([g]) == {autotune.shape_key(g): 8}
