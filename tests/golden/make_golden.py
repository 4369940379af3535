"""Generates tests/golden/refpin_*.npz: outputs of the reference's OWN device functions and host
classes (host-compiled from the reference tree by oracle/ref_pin) on small seeded inputs.

Run in a container that has the reference sources:  python tests/golden/make_golden.py
The fixtures pin the oracle where the reference tree is absent (e.g. on the GPU machine).
"""
import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)

from oracle.ref_pin import refpin  # noqa: E402
from steadyscan_b200 import prep, synth  # noqa: E402

CASES = {
    # name: (nlines, linewidth, nknots, n_frames, settings extras, groupsize)
    "uniform_even": (16, 12, 5, 4, {}, 2),
    "uniform_odd": (16, 12, 5, 3, {}, 2),
    "nonint_lines_per_knot": (18, 10, 6, 3, {}, 2),
    "bidirectional_k1": (12, 10, 13, 2, {"isbidirectional": True}, 2),
    "cropped": (16, 14, 5, 3, {"cropping": [1, 2, 0, 0]}, 1),
}


def make_case(name, seed=123):
    nl, lw, nk, nF, extra, gsz = CASES[name]
    rec = synth.make_recording(nl, lw, nF, nk, n_blobs=6, sigma=(1.5, 3.0), walk_sigma=0.3, clip_px=2.5,
                               jumps_per_frame=1, jump_px=1.5, seed=seed)
    st = dict(nknots=nk, gpu_frame_groupsize=gsz)
    st.update(extra)
    s = prep.init_settings(st, rec.template, nl, lw)
    lay = prep.block_layout(s)
    bm = prep.frames_to_blockmatrix(rec.frames, lay)
    args = prep.boundary_arguments(s, rec.template, bm, nF, layout=lay)
    return args


def knots(args, seed):
    rng = np.random.default_rng(seed)
    w = args["tfrac"].shape[1]
    N = w * int(args["nFrames"]) + 1
    p = rng.normal(0.0, 1.2, 2 * N)
    p[0:2] += 40.0      # a few knots far outside the template
    p[N + 3] -= 30.0
    return p


def main():
    out_dir = os.path.dirname(os.path.abspath(__file__))
    for name in CASES:
        args = make_case(name)
        store = {f"in_{k}": np.asarray(v) for k, v in args.items() if k != "flags"}
        store["in_flags"] = np.array(args["flags"])
        for shift in (0, 1):
            p = knots(args, 10 + shift)
            r = refpin.assemble(args, p, shift)
            store[f"s{shift}_p"] = p
            for k in ("x", "y", "mask", "diff", "wx", "wy", "params_used", "blocks_present", "offsets", "jtr",
                      "errval"):
                store[f"s{shift}_{k}"] = r[k]
            valid = r["hr"] != np.iinfo(np.int32).max
            store[f"s{shift}_coo_slot"] = np.nonzero(valid)[0].astype(np.int32)
            store[f"s{shift}_coo_row"] = r["hr"][valid]
            store[f"s{shift}_coo_col"] = r["hc"][valid]
            store[f"s{shift}_coo_val"] = r["hv"][valid]
            store[f"s{shift}_n_used"] = np.array(r["n_used"])
            rng = np.random.default_rng(20 + shift)
            ndp = rng.normal(0, 1, p.size)
            dp0 = rng.normal(0, 1, p.size)
            store[f"s{shift}_expand_new"] = ndp
            store[f"s{shift}_expand_old"] = dp0
            store[f"s{shift}_expand_out"] = refpin.expand(args, p, shift, r["params_used"], r["offsets"], ndp, dp0)
            gc, _ = refpin.global_corr(args, r["mask"], r["diff"])
            store[f"s{shift}_global_corr"] = np.array(gc)
        w = args["tfrac"].shape[1]
        nF = int(args["nFrames"])
        rng = np.random.default_rng(5)
        px = rng.normal(0, 1, (w + 1) * nF)
        py = rng.normal(0, 1, (w + 1) * nF)
        store["org_px"], store["org_py"] = px, py
        store["org_p"] = refpin.organize2d1(px, py, nF, w)
        store["org_back_x"], store["org_back_y"] = refpin.organize1d2(store["org_p"], nF, w)
        v = rng.normal(0, 1, 37)
        store["filt_in"] = v
        store["filt_smear"] = refpin.smearing_filter(v, 0.8)
        store["filt_range"] = refpin.range_filter(v, 0.8)
        np.savez_compressed(os.path.join(out_dir, f"refpin_{name}.npz"), **store)
        print("wrote", name)


if __name__ == "__main__":
    main()
