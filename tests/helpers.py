"""Shared builders for the tests: small seeded align_group_to_template problems."""
from __future__ import annotations

import numpy as np

from steadyscan_b200 import prep, synth


def make_args(nlines=32, linewidth=32, nknots=9, n_frames=4, seed=3, n_blobs=10, sigma=(1.5, 3.5), walk_sigma=0.15,
              clip_px=3.0, jumps=1, jump_px=2.0, frame_dtype=np.float64, settings=None, template_size=None,
              noise=True):
    """A recording and its 26 boundary arguments (dict). ``settings`` overrides the defaults."""
    th, tw = template_size or (nlines, linewidth)
    rec = synth.make_recording(th, tw, n_frames, nknots, n_blobs=n_blobs, sigma=sigma, walk_sigma=walk_sigma,
                               clip_px=clip_px, jumps_per_frame=jumps, jump_px=jump_px, seed=seed,
                               nlines=nlines, linewidth=linewidth, noise=noise)
    st = {"nknots": nknots}
    st.update(settings or {})
    s = prep.init_settings(st, rec.template, nlines, linewidth)
    lay = prep.block_layout(s)
    frames = rec.frames_as(frame_dtype)
    bm = prep.frames_to_blockmatrix(frames, lay, dtype=frame_dtype)
    args = prep.boundary_arguments(s, rec.template, bm, n_frames, layout=lay)
    return args, rec, s


def knot_rms(a, b):
    return float(np.sqrt(np.mean((np.asarray(a) - np.asarray(b)) ** 2)))
