"""Generates tests/golden/refrun_*.npz: whole align_group_to_template runs of the reference's OWN
task layer (Task::alignFrames, MainIteration::execute, the kernels and their launchers, the filters,
ParameterOrganizer and SolverCuSolver), host-compiled from the reference tree by oracle/ref_pin
(run_transform.py, hostcuda.*, refrun.cpp), on small seeded groups.

Run in a container that has the reference sources:  python tests/golden/make_refrun_golden.py
Each fixture holds the 26 inputs and the run's outputs: iterations, stop reason, per-frame knots,
frame correlations, residrms, the mask, the knot chain after every iteration and (flags C and e)
every iteration's global correlation and every half-step's errvals, and (flag t) the chain after
every half-step. The cases keep frames of at
most 32 blocks, so that a frame's line-search block is one warp, whose lock-step execution the
host emulation reproduces; the solver is id 1 (exact Cholesky: Eigen, the default id 2, is not
part of the reference tree). Flag R is left out: its median kernel (d_medianfilter.cu:3-20) reads
before and after the array it filters and filters in place across threads, which the oracle and the
CUDA path replace by an out-of-place filter that keeps both ends.
"""
import os
import sys

import numpy as np

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), "..", ".."))
sys.path.insert(0, ROOT)

from oracle.ref_pin import refpin  # noqa: E402
from tests.helpers import make_args  # noqa: E402

CASES = {
    # name: (make_args keywords, flags)
    "smearing_default": (dict(seed=3, settings={"gpu_solver_id": 1}), "DCce"),
    "range_filter": (dict(seed=4, settings={"gpu_solver_id": 1, "gpu_filter_id": 2}), "DCce"),
    "no_filter": (dict(seed=5, settings={"gpu_solver_id": 1, "gpu_filter_id": 0}), "DCce"),
    "odd_frames": (dict(n_frames=3, seed=6, settings={"gpu_solver_id": 1}), "DCce"),
    "big_motion": (dict(clip_px=6.0, jumps=2, jump_px=4.0, seed=11, settings={"gpu_solver_id": 1}), "DCce"),
    "nonint_lines_per_knot": (dict(nlines=30, linewidth=20, nknots=8, seed=7, settings={"gpu_solver_id": 1}), "DCce"),
    "bidirectional_k1": (dict(nlines=16, linewidth=16, nknots=17, seed=26,
                              settings={"gpu_solver_id": 1, "isbidirectional": True}), "DCce"),
    "mask_inactive": (dict(n_frames=4, seed=9, settings={"gpu_solver_id": 1, "haltcorr": 0.9}), "DCceM"),
    # frames inactive over consecutive iterations (flag c's frame correlations are low, so a low
    # haltcorr deactivates them): their difference-image buffers are swapped by several global
    # correlations without being rewritten
    "mask_inactive_stale": (dict(n_frames=6, seed=16, settings={"gpu_solver_id": 1, "haltcorr": 0.2}), "DCceM"),
    "mask_inactive_stale_b": (dict(n_frames=6, seed=10, settings={"gpu_solver_id": 1, "haltcorr": 0.15}), "DCceM"),
    # 40 frames of 8 blocks: fW = 320 columns, so the global correlation's swap-back (the first
    # 512 pixels in row-major order) ends inside the second row
    "swap_back_row1": (dict(n_frames=40, seed=33, settings={"gpu_solver_id": 1}), "DCce"),
    "frames_32_blocks": (dict(nlines=64, linewidth=24, nknots=33, n_frames=4, seed=12,
                              settings={"gpu_solver_id": 1}), "DCce"),
    # huge first steps: a trial with no block present whose moving knots belong to the frame's first
    # threads (the block-wide movement flag after such a trial)
    "absent_trial_movement": (dict(seed=45, n_frames=4, clip_px=6.0, jumps=2, jump_px=4.0,
                                   settings={"gpu_solver_id": 1, "gpu_filter_max_iterations": 2}), "DCce"),
    # flag t (TimedMainIteration): the retry without filter as iteration + 1, paramsUsed cleared
    # before every half-step (with the odd frame count's inactive last group), the filterID rules
    # that move the filter-deactivation branch, and rgParams
    "timed_retry_odd": (dict(n_frames=3, seed=6, settings={"gpu_solver_id": 1}), "DCcet"),
    "timed_filter_limit": (dict(seed=41, n_frames=4, clip_px=6.0, jumps=2, jump_px=4.0,
                                settings={"gpu_solver_id": 1, "gpu_filter_max_iterations": 2}), "DCcet"),
    "timed_mask_inactive": (dict(n_frames=6, seed=10, settings={"gpu_solver_id": 1, "haltcorr": 0.15}), "DCceMt"),
}


def main():
    out_dir = os.path.dirname(os.path.abspath(__file__))
    for name, (kw, flags) in CASES.items():
        args, _, _ = make_args(**kw)
        args["flags"] = flags
        assert args["tfrac"].shape[1] <= 32, "one warp per frame's line-search block"
        r = refpin.run_align(args)
        # a solve of a matrix that is not positive definite leaves the step unspecified (cuSOLVER's
        # report is ignored by the reference): such a run pins nothing
        assert r["singular_solves"] == 0, f"{name}: {r['singular_solves']} non-SPD solves"
        it = int(r["iterations"])
        store = {f"in_{k}": np.asarray(v) for k, v in args.items() if k != "flags"}
        store["in_flags"] = np.array(args["flags"])
        store["iterations"] = np.array(it)
        store["stop_reason"] = np.array(r["stop_reason"])
        for k in ("dx", "dy", "frame_corr", "residrms", "mask"):
            store[k] = r[k]
        store["all_params"] = r["all_params"][:it]
        store["iter_corr"] = r["iter_corr"][:it]
        store["iter_errvals"] = r["iter_errvals"][:2 * it]
        store["frame_corr_hist"] = r["frame_corr_hist"][:it]
        if "t" in flags:  # the slots a run writes: two per iteration, two more for a last retry
            store["rg_params"] = r["rg_params"][:2 * it + 2]
        np.savez_compressed(os.path.join(out_dir, f"refrun_{name}.npz"), **store)
        print("wrote", name, "iterations", it, "stop", r["stop_reason"])


if __name__ == "__main__":
    main()
