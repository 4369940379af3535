"""Autotuner of the evaluation tile schedule: frames per tile, per group shape.

The assembly, trial-round, correlation and final kernels run one CTA per tile, a tile being one
block column of ``frames_per_cta`` consecutive frames of a group (``ss_inputs.frames_per_cta``; 0
splits a group into even chunks of at most 32 frames). Few frames per tile give many small CTAs,
each staging its own template row window; many frames per tile give fewer CTAs that reuse one
window over more frames but fill fewer SMs. The best split depends on the block height (pixels per
block column), the number of block columns, the frame storage type and the precision, so the tuner
picks it per shape by timing the candidates on the caller's own groups:

* groups are keyed by (block height, block columns, template shape, frame type, precision, template
  storage, caller-given gradients);
* for a key not yet tuned, up to ``probe_groups`` of its groups (at most ``probe_frames`` frames in
  all), repeated until the batch has ``min_tiles`` tiles at the default split (so that, as inside a
  large ragged batch, the GPU is full and the time measures throughput rather than latency), run as
  one batch per candidate, ``reps`` timed runs after one warm-up, and the candidate with the lowest
  median time wins (the tile split changes no precision-D result and precision-S results
  only at FP32 rounding level, so every candidate does essentially the same iterations);
* choices are kept per tuner and, with ``cache_path``, in a JSON file keyed by device name;
* ``apply(..., validate=True)`` then times the caller's whole batch once with the tuned split and once
  with the default split and keeps the faster (per-shape timing misses interactions between shapes
  that share the GPU in one batch); ``last_validation`` records both times.

The reference has no counterpart (its kernels use fixed launch shapes, task_*.cu).
"""
from __future__ import annotations

import json
import os
import time

import numpy as np

from . import api

CANDIDATES = (4, 8, 16, 32, 64)


def _frame_type(a: dict) -> str:
    d = a["bmData"]
    if isinstance(d, api.DeviceMatrix):
        return f"dev{d.dtype}"
    return np.asarray(d).dtype.str


def _gradients_given(a: dict) -> bool:
    """True when xgrad / ygrad are not the template's forward differences (the library then samples
    separate gradient quads and stages no template windows, a different per-pixel cost)."""
    if "xgrad" not in a or "ygrad" not in a:
        return False
    t = np.asarray(a["template_image"], dtype=np.float64)
    xg, yg = np.asarray(a["xgrad"], dtype=np.float64), np.asarray(a["ygrad"], dtype=np.float64)
    if xg.shape != t.shape or yg.shape != t.shape:
        return True
    return not (np.array_equal(xg[:, :-1], np.diff(t, axis=1)) and np.array_equal(yg[:-1, :], np.diff(t, axis=0)))


def shape_key(a: dict, template_storage=None) -> str:
    """The tuning key of one group's argument dict: block height and columns, template shape, frame
    type, precision, template storage and whether the gradients are the caller's own. Settings that
    change how many iterations a group runs but not the work of one evaluation tile (filters,
    lambda, thresholds, iteration limits) are not part of the key."""
    tf = np.asarray(a["tfrac"])
    flags = a["flags"] if isinstance(a["flags"], str) else bytes(a["flags"]).decode()
    prec = "S" if "S" in flags else "D"
    th, tw = np.asarray(a["template_image"]).shape
    grads = "_gq" if _gradients_given(a) else ""
    return f"hb{tf.shape[0]}_w{tf.shape[1]}_t{th}x{tw}_{_frame_type(a)}_{prec}_{template_storage or 'f32'}{grads}"


def _device_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name()
    except Exception:  # pragma: no cover - no torch device
        return "unknown"


class Autotuner:
    def __init__(self, cache_path: str | None = None, candidates=CANDIDATES, reps: int = 3, probe_groups: int = 4,
                 probe_frames: int = 256, min_tiles: int = 4096, max_repeat: int = 16):
        self.cache_path = cache_path
        self.candidates = tuple(int(c) for c in candidates)
        self.reps = int(reps)
        self.probe_groups = int(probe_groups)
        self.probe_frames = int(probe_frames)
        self.min_tiles = int(min_tiles)
        self.max_repeat = int(max_repeat)
        self.choices: dict = {}
        self.timings: dict = {}
        self.last_validation: dict | None = None
        self._device = _device_name()
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                self.choices.update(json.load(f).get(self._device, {}))

    def _save(self):
        if not self.cache_path:
            return
        data = {}
        if os.path.exists(self.cache_path):
            with open(self.cache_path) as f:
                data = json.load(f)
        data.setdefault(self._device, {}).update(self.choices)
        tmp = self.cache_path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, self.cache_path)

    def _probe(self, groups: list) -> list:
        """Up to probe_groups groups with at most probe_frames frames in all (the largest first)."""
        order = sorted(range(len(groups)), key=lambda i: -int(groups[i]["nFrames"]))
        out, n = [], 0
        for i in order:
            nf = int(groups[i]["nFrames"])
            if out and n + nf > self.probe_frames:
                continue
            out.append(groups[i])
            n += nf
            if len(out) >= self.probe_groups:
                break
        # tiles at the default split: block columns x chunks of at most 32 frames
        tiles = sum(np.asarray(g["tfrac"]).shape[1] * -(-int(g["nFrames"]) // 32) for g in out)
        rep = min(self.max_repeat, max(1, -(-self.min_tiles // max(1, tiles))))
        return out * rep

    def _time(self, probe: list, fpc, template_storage) -> float:
        """Median seconds of one run of ``probe`` at frames_per_cta ``fpc`` (an int for every group,
        or None to keep each group's own)."""
        gs = probe if fpc is None else [dict(g, frames_per_cta=fpc) for g in probe]
        b = api.Batch(gs, template_storage=template_storage)
        try:
            b.run()  # warm-up: graph capture, attributes, caches
            ts = []
            for _ in range(self.reps):
                t0 = time.perf_counter()
                b.run()
                ts.append(time.perf_counter() - t0)
        finally:
            b.close()
        return float(np.median(ts))

    def tune(self, groups: list, template_storage=None) -> dict:
        """Tunes every key of ``groups`` not yet chosen; returns {key: frames_per_cta}."""
        by_key: dict = {}
        for g in groups:
            by_key.setdefault(shape_key(g, template_storage), []).append(g)
        changed = False
        for key, gs in by_key.items():
            if key in self.choices:
                continue
            probe = self._probe(gs)
            most = max(int(g["nFrames"]) for g in probe)
            # a tile holds at most the group's frames: larger candidates repeat the largest useful one
            cands = [c for c in self.candidates if c <= most] or [min(self.candidates)]
            if most < max(self.candidates) and most not in cands and most > cands[-1]:
                cands.append(most)
            t = {c: self._time(probe, c, template_storage) for c in cands}
            best = min(t, key=t.get)
            self.timings[key] = t
            self.choices[key] = int(best)
            changed = True
        if changed:
            self._save()
        return {k: self.choices[k] for k in by_key}

    def apply(self, groups: list, template_storage=None, validate: bool = False) -> list:
        """Copies of ``groups`` with the tuned frames_per_cta (tuning the keys not yet chosen); with
        ``validate``, the default split instead when it runs the whole batch faster."""
        self.tune(groups, template_storage)
        tuned = [dict(g, frames_per_cta=self.choices[shape_key(g, template_storage)]) for g in groups]
        if not validate:
            return tuned
        t_tuned = self._time(tuned, None, template_storage)
        t_default = self._time(groups, 0, template_storage)
        self.last_validation = {"tuned_s": t_tuned, "default_s": t_default, "kept": "tuned"}
        if t_default < t_tuned:
            self.last_validation["kept"] = "default"
            return [dict(g, frames_per_cta=0) for g in groups]
        return tuned
