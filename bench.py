"""Benchmark of the batched align_group_to_template path on B200.

Workload (default): 2000 synthetic 512x512 uint16 frames (400-blob template, per-line random-walk
motion with jumps, Poisson noise at a 200-photon peak), knots every 2 lines (257 knots per frame),
aligned in groups of 64 frames, precision 'S' (FP32 pixel arithmetic, FP64 reduction and solve),
lambda 5e-3, default settings otherwise. One step aligns all frames, every group from its initial
knots to its stop criterion.

  value   frames/s with the frames already resident in HBM (CUDA events on the engine's stream)
  e2e     frames/s through the public C ABI (ss_align_groups) from pinned host buffers, host->device
          and device->host copies inside the timed region
Prints ONE JSON line (rank 0). ``--impl reference`` times the reference algorithm's CPU
restatement on a bounded sample of the same workload instead.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "frames/s at 512², 2-line knots; p99 group latency vs plain GPU, ≤0.05px vs FP64"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--frames", type=int, default=2000)
    ap.add_argument("--group", type=int, default=64)
    ap.add_argument("--size", type=int, default=512)
    ap.add_argument("--precision", default="S", choices=["S", "D"])
    ap.add_argument("--cpu-sample-frames", type=int, default=16)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the unbatched per-group comparison")
    ap.add_argument("--no-sweep", action="store_true", help="skip the storage-precision sweep")
    ap.add_argument("--cpu-single-frames", type=int, default=4,
                    help="frames of the single-thread CPU baseline (0: skip it)")
    ap.add_argument("--sweep-frames", type=int, default=4000,
                    help="frames of the storage sweep on the device (0: skip it)")
    ap.add_argument("--no-pipeline", action="store_true",
                    help="skip the frame preparation and reconstruction legs")
    ap.add_argument("--recon-frames", type=int, default=64, help="frames of the reconstruction leg")
    ap.add_argument("--plain-groups", type=int, default=2)
    ap.add_argument("--serve-seconds", type=float, default=60.0,
                    help="seconds of generated serving load (8 sessions, 0 to skip)")
    ap.add_argument("--ragged-groups", type=int, default=0, help="groups of the ragged batch (0: 96)")
    ap.add_argument("--ragged-single", type=int, default=16,
                    help="groups of the ragged batch also run one batch per group")
    ap.add_argument("--no-ragged", action="store_true", help="skip the ragged batch with the autotuner")
    ap.add_argument("--only-ragged", action="store_true", help="run and print only the ragged batch")
    ap.add_argument("--only-pipeline", action="store_true",
                    help="run and print only the frame preparation and reconstruction legs")
    ap.add_argument("--ragged-lean", action="store_true",
                    help="ragged batch at the default schedule only (no tuner, no comparison runs)")
    ap.add_argument("--serve-warm", action="store_true",
                    help="start each session's groups from its last displacement instead of zero")
    return ap.parse_args()


# ------------------------------------------------------------------------------------------------
# workload

def to_block_columns(img, k):
    """A frame (lines x pixels tensor) as a flat block matrix of the default scan geometry: block
    column cc holds lines cc*k .. cc*k+k-1, MATLAB column-major inside the block."""
    nlines, linewidth = img.shape
    return img.view(nlines // k, k, linewidth).permute(0, 2, 1).contiguous().view(-1)


def render_block_frames(tmpl, walk, n_frames, nlines, linewidth, k, gen, device):
    """uint16 frames (Poisson counts of the template sampled along ``walk``, one row per scan line),
    each as a flat block matrix: block column cc holds lines cc*k .. cc*k+k-1, MATLAB column-major
    inside the block."""
    import torch
    T = tmpl if isinstance(tmpl, torch.Tensor) else torch.tensor(tmpl, device=device)
    th, tw = T.shape
    jj = torch.arange(linewidth, device=device, dtype=torch.float64)[None, :]
    ll = torch.arange(nlines, device=device, dtype=torch.float64)[:, None]
    wl_all = walk if isinstance(walk, torch.Tensor) else torch.tensor(walk, device=device)
    bg = float(T.min())
    out = []
    for f in range(n_frames):
        wl = wl_all[f * nlines:(f + 1) * nlines]
        x = jj + wl[:, 0:1]
        y = ll + wl[:, 1:2]
        x0 = torch.floor(x)
        y0 = torch.floor(y)
        fx, fy = x - x0, y - y0
        x0l, y0l = x0.long(), y0.long()
        inside = (x0l >= 0) & (y0l >= 0) & (x0l < tw - 1) & (y0l < th - 1)
        xc, yc = x0l.clamp(0, tw - 2), y0l.clamp(0, th - 2)
        v = (1 - fx) * ((1 - fy) * T[yc, xc] + fy * T[yc + 1, xc]) + fx * ((1 - fy) * T[yc, xc + 1] + fy * T[yc + 1, xc + 1])
        lam = torch.where(inside, v, torch.full_like(v, bg))
        cnt = torch.poisson(lam, generator=gen).clamp(0, 65535).to(torch.int32).to(torch.uint16)
        out.append(to_block_columns(cnt, k))
    return out


def make_workload(n_frames, size, group, precision, seed, device):
    """Returns (groups: list of host argument dicts, device frame tensors per group, settings)."""
    import torch

    from steadyscan_b200 import prep, synth
    rng = np.random.default_rng(seed)
    nk = size // 2 + 1
    # column-major, as the C ABI reads it: no conversion per call
    tmpl = np.asfortranarray(synth.make_template(size, size, 400 * (size * size) // (512 * 512), (2.0, 6.0), rng))
    walk = synth.make_walk(size * (n_frames + 1), 0.1, 10.0, (0, 3), size, 4.0, rng)
    s = prep.init_settings({"nknots": nk, "gpu_forced_precision": precision, "lambda": 5e-3}, tmpl, size, size)
    lay = prep.block_layout(s)
    k = size // (nk - 1)
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    frames_bm = render_block_frames(tmpl, walk, n_frames, size, size, k, gen, device)
    groups, dev = [], []
    grads = prep.template_gradients(tmpl)
    for g0 in range(0, n_frames, group):
        nF = min(group, n_frames - g0)
        flat = torch.cat(frames_bm[g0:g0 + nF])
        dev.append(flat)
        host = flat.cpu().numpy().reshape(lay.frame_h, lay.frame_w * nF, order="F")
        args = prep.boundary_arguments(s, tmpl, host, nF, layout=lay, gradients=grads)
        groups.append(args)
    return groups, dev, s, lay


def plain_small(device, threads):
    """The plain-method small workload: 50 uint16 frames of a 256x256 template (80 blobs, sigma 2-5
    px), walk N(0, 0.15 px/line) clipped to +-6 px with one jump of up to 4 px per frame, Poisson
    noise, knots every 4 lines (65 knots), lambda 1e-2, at most 30 iterations. The FP64 CPU
    restatement on all host threads against one GPU call in precision D and in precision S."""
    import torch

    from oracle import oracle
    from steadyscan_b200 import api, prep, synth
    sp = synth.WORKLOADS[1]
    rng = np.random.default_rng(sp["seed"])
    h, w, nf, nk = sp["h"], sp["w"], sp["n_frames"], sp["nknots"]
    tmpl = synth.make_template(h, w, sp["n_blobs"], sp["sigma"], rng)
    walk = synth.make_walk(h * (nf + 1), sp["walk_sigma"], sp["clip_px"], sp["jumps_per_frame"], h, sp["jump_px"], rng)
    s = prep.init_settings({"nknots": nk, "lambda": sp["lam"], "max_iter": sp["max_iter"]}, tmpl, h, w)
    lay = prep.block_layout(s)
    gen = torch.Generator(device=device)
    gen.manual_seed(sp["seed"])
    flat = torch.cat(render_block_frames(tmpl, walk, nf, h, w, h // (nk - 1), gen, device))
    host = flat.cpu().numpy().reshape(lay.frame_h, lay.frame_w * nf, order="F")
    a = prep.boundary_arguments(s, tmpl, host, nf, layout=lay)
    oracle.build()
    t0 = time.perf_counter()
    o = oracle.align_group(dict(a, flags="D"), n_threads=threads, want_mask=False)
    cpu_s = time.perf_counter() - t0
    out = {"workload": "50 frames 256x256 uint16, knots every 4 lines (65 knots), lambda 1e-2, at most 30 "
                       "iterations", "fp64_oracle": {"frames_per_s": nf / cpu_s, "cores": threads,
                                                     "iterations": int(o["iterations"])}}
    ref = np.concatenate([o["dx"], o["dy"]])
    for prec in ("D", "S"):
        api.align_group(dict(a, flags=prec), want_mask=False)  # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g = api.align_group(dict(a, flags=prec), want_mask=False)
        dt = time.perf_counter() - t0
        e = np.concatenate([g["dx"], g["dy"]]) - ref
        out[prec] = {"frames_per_s_one_call": nf / dt, "iterations": int(g["iter_used"]),
                     "rms_px_vs_fp64_oracle": float(np.sqrt(np.mean(e * e))),
                     "max_px_vs_fp64_oracle": float(np.max(np.abs(e)))}
    return out


RAGGED_SETTINGS = {"lambda": 1e-2, "move_thresh": 1e-3, "max_iter": 30}


def make_ragged_workload(precision, seed, device, n_groups=None, walks=None):
    """Ragged batch: groups of U[1,128] frames, each of a frame size drawn from 128x128, 256x512,
    512x512 and 796x512 (lines x pixels) and a knot spacing from {1, 2, 4} lines; one template per
    frame size (80 blobs per 256x256 of area, sigma 2-5 px, 200-photon peak); per-line random walk
    N(0, 0.15 px) clipped to +-6 px with one jump of up to 4 px per frame; Poisson noise; lambda
    1e-2, move threshold 1e-3 px, at most 30 iterations. Returns (host argument dicts, device frame
    tensors, per-group (lines, pixels, lines per knot, frames)); a list ``walks`` receives each
    group's per-line displacement (the ground truth)."""
    import torch

    from steadyscan_b200 import prep, synth
    sp = synth.WORKLOADS[3]
    rng = np.random.default_rng(seed)
    n_groups = n_groups or sp["n_groups"]
    gen = torch.Generator(device=device)
    gen.manual_seed(seed)
    tmpls, setts = {}, {}
    groups, dev, meta = [], [], []
    for _ in range(n_groups):
        h, w = sp["sizes"][int(rng.integers(len(sp["sizes"])))]
        k = sp["lines_per_knot"][int(rng.integers(len(sp["lines_per_knot"])))]
        nf = int(rng.integers(sp["group_len"][0], sp["group_len"][1] + 1))
        if (h, w) not in tmpls:
            t = synth.make_template(h, w, max(1, round(80 * h * w / (256 * 256))), (2.0, 5.0), rng)
            tmpls[(h, w)] = (t, prep.template_gradients(t), torch.tensor(t, device=device))
        tmpl, grads, tdev = tmpls[(h, w)]
        if (h, w, k) not in setts:
            s = prep.init_settings(dict(RAGGED_SETTINGS, nknots=h // k + 1, gpu_forced_precision=precision), tmpl, h, w)
            setts[(h, w, k)] = (s, prep.block_layout(s))
        s, lay = setts[(h, w, k)]
        walk = synth.make_walk(h * (nf + 1), sp["walk_sigma"], sp["clip_px"], sp["jumps_per_frame"], h,
                               sp["jump_px"], rng)
        if walks is not None:
            walks.append(walk)
        flat = torch.cat(render_block_frames(tdev, walk, nf, h, w, k, gen, device))
        host = flat.cpu().numpy().reshape(lay.frame_h, lay.frame_w * nf, order="F")
        groups.append(prep.boundary_arguments(s, tmpl, host, nf, layout=lay, gradients=grads))
        dev.append((flat, lay))
        meta.append((h, w, k, nf))
    return groups, dev, meta


def device_groups(groups, dev):
    """Argument dicts whose frames are the device tensors (uint16 block matrices)."""
    from steadyscan_b200 import api
    from steadyscan_b200._lib import SS_U16
    out = []
    for g, (t, lay) in zip(groups, dev):
        d = dict(g)
        d["bmData"] = api.DeviceMatrix(t.data_ptr(), lay.frame_h, lay.frame_w * int(g["nFrames"]), SS_U16, owner=t)
        out.append(d)
    return out


def timed_batch(groups, device, steps, warmup=1, graph=True, template_storage=None):
    """Device ms per run of one batch (CUDA events on the engine's stream), its stats and results."""
    import torch

    from steadyscan_b200 import api
    b = api.Batch(groups, template_storage=template_storage)
    b.set_graph(graph)
    stream = torch.cuda.ExternalStream(b.stream_ptr, device=device)
    for _ in range(warmup):
        b.run()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    launches = 0
    for _ in range(steps):
        b.run()
        launches += b.stats()["kernel_launches"]
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    st = b.stats()
    res = b.collect()
    b.close()
    return ms, st, res, launches


def ragged(args, device):
    """The ragged batch with the autotuned tile schedule, as one graph launch per run, next to the
    default schedule, host-launched cycles, one batch per group, and the FP64 path."""
    from steadyscan_b200 import synth
    from steadyscan_b200.autotune import Autotuner
    walks = []
    groups, dev, meta = make_ragged_workload("S", 1003, device, args.ragged_groups or None, walks=walks)
    dg = device_groups(groups, dev)
    frames = sum(m[3] for m in meta)
    steps = max(1, args.steps)
    if args.ragged_lean:
        ms, st, res, launches = timed_batch(dg, device, steps, warmup=args.warmup)
        iters = np.array([r["iter_used"] for r in res])
        # per-pass device time from one run with event timing (host-launched cycles)
        from steadyscan_b200 import api
        b = api.Batch(dg)
        b.set_timing(True)
        b.run()
        rs = b.stats()
        b.close()
        return {"frames": frames, "groups": len(meta), "value": frames / (ms / 1e3), "unit": "frames/s",
                "ms_per_run": ms, "kernel_launches_per_run": launches // steps, "cycles": st["cycles"],
                "linesearch_rounds": st["linesearch_rounds"],
                "iterations": {"min": int(iters.min()), "max": int(iters.max()), "mean": float(iters.mean())},
                "timed_run": {"run_ms": rs["run_ms"], "cycles": rs["cycles"], "rounds": rs["linesearch_rounds"],
                              "eval_ms": dict(zip(("assembly", "trial", "correlation", "final"), rs["eval_ms"])),
                              "frame_passes": dict(zip(("assembly", "trial", "correlation", "final"),
                                                       rs["frame_passes"]))}}
    tuner = Autotuner(candidates=(8, 16, 32, 64), reps=2)
    t0 = time.perf_counter()
    tuned = tuner.apply(dg, validate=True)
    tune_s = time.perf_counter() - t0
    ms_t, st_t, res_t, launches = timed_batch(tuned, device, steps)
    ms_d, st_d, res_d, _ = timed_batch(dg, device, steps)
    ms_h, st_h, res_h, _ = timed_batch(tuned, device, steps, graph=False)
    # graph and host-launched cycles agree bit for bit; tile schedules at FP32 rounding level
    same = all(np.array_equal(a["dx"], b["dx"]) and np.array_equal(a["dy"], b["dy"]) for a, b in zip(res_t, res_h))
    sched_diff = max(float(np.max(np.abs(np.concatenate([a["dx"] - b["dx"], a["dy"] - b["dy"]]))))
                     for a, b in zip(res_t, res_d))
    # one batch per group, serially (a sample of the groups)
    n1 = min(len(tuned), args.ragged_single)
    ms1, fr1 = 0.0, 0
    for g in tuned[:n1]:
        ms, _, _, _ = timed_batch([g], device, 1)
        ms1 += ms
        fr1 += int(g["nFrames"])
    # FP64 reference: precision D on the same frames (the D path agrees with the FP64 oracle to 1e-6 px)
    dgd = [dict(g, flags="D") for g in dg]
    ms_64, _, res_64, _ = timed_batch(dgd, device, 1, warmup=0)
    # error of precision S against FP64 per frame size: over all knots, and over the knots where the
    # FP64 solution is within 0.5 px of the true displacement (elsewhere the problem is ill-posed,
    # e.g. knots every line on lines without template structure, and FP64 itself runs away from the
    # truth, so tiny rounding differences grow); knots within 0.5 px of the truth for both precisions
    acc = {}
    for (h, w, k, nf), wk, a, o in zip(meta, walks, res_t, res_64):
        nk = h // k + 1
        tx, ty = synth.truth_knots(wk, h, nk, nf)
        sx, sy = np.asarray(a["dx"]).reshape(nf, nk).T, np.asarray(a["dy"]).reshape(nf, nk).T
        ox, oy = np.asarray(o["dx"]).reshape(nf, nk).T, np.asarray(o["dy"]).reshape(nf, nk).T
        e = np.concatenate([(sx - ox).ravel(), (sy - oy).ravel()])
        e = e[np.isfinite(e)]
        # the last knot of a frame repeats the one before it (an output convention), not a time point
        inner = np.zeros_like(tx, dtype=bool)
        inner[:-1] = True
        ok64 = inner & (np.abs(ox - tx) <= 0.5) & (np.abs(oy - ty) <= 0.5)
        okS = inner & (np.abs(sx - tx) <= 0.5) & (np.abs(sy - ty) <= 0.5)
        ec = np.concatenate([(sx - ox)[ok64], (sy - oy)[ok64]])
        # the frames the reference's caller keeps (steady_scan.m:246-284), from the FP64 run:
        # correlation >= corr_thresh 0.75 and >= minblockfrac 0.25 of the blocks with a valid pixel
        keep = (np.asarray(o["frame_corr"]) >= 0.75) & (np.asarray(o["blocks_used"]).mean(axis=0) >= 0.25)
        ea = np.concatenate([(sx - ox)[:, keep].ravel(), (sy - oy)[:, keep].ravel()])
        ea = ea[np.isfinite(ea)]
        cur = acc.setdefault(f"{h}x{w}", {"se": 0.0, "n": 0, "max": 0.0, "se_c": 0.0, "n_c": 0, "max_c": 0.0,
                                          "knots": 0, "ok64": 0, "okS": 0, "se_a": 0.0, "n_a": 0, "max_a": 0.0,
                                          "frames": 0, "kept": 0})
        cur["se_a"] += float(np.sum(ea * ea))
        cur["n_a"] += ea.size
        cur["max_a"] = max(cur["max_a"], float(np.max(np.abs(ea))) if ea.size else 0.0)
        cur["frames"] += nf
        cur["kept"] += int(keep.sum())
        cur["se"] += float(np.sum(e * e))
        cur["n"] += e.size
        cur["max"] = max(cur["max"], float(np.max(np.abs(e))))
        cur["se_c"] += float(np.sum(ec * ec))
        cur["n_c"] += ec.size
        cur["max_c"] = max(cur["max_c"], float(np.max(np.abs(ec))) if ec.size else 0.0)
        cur["knots"] += int(inner.sum())
        cur["ok64"] += int(ok64.sum())
        cur["okS"] += int(okS.sum())
    err = {k: {"rms_px": float(np.sqrt(v["se"] / v["n"])), "max_px": v["max"],
               "rms_px_where_fp64_within_0.5px_of_truth": float(np.sqrt(v["se_c"] / max(1, v["n_c"]))),
               "max_px_where_fp64_within_0.5px_of_truth": v["max_c"],
               "knots_within_0.5px_of_truth": {"fp64": v["ok64"] / v["knots"], "S": v["okS"] / v["knots"]},
               "frames_kept_by_the_caller": f"{v['kept']} of {v['frames']}",
               "rms_px_kept_frames": float(np.sqrt(v["se_a"] / max(1, v["n_a"]))),
               "max_px_kept_frames": v["max_a"]}
           for k, v in acc.items()}
    iters = np.array([r["iter_used"] for r in res_t])
    choices = {k: v for k, v in tuner.choices.items()}
    timings = {k: {str(c): round(1e3 * t, 3) for c, t in v.items()} for k, v in tuner.timings.items()}
    return {"workload": f"{len(meta)} groups, U[1,128] frames of 128x128 / 256x512 / 512x512 / 796x512 "
                        "uint16, knots every 1, 2 or 4 lines, precision S, lambda 1e-2, move threshold 1e-3 px, "
                        "at most 30 iterations",
            "frames": frames, "groups": len(meta),
            "frames_by_size": {k: int(sum(m[3] for m in meta if f"{m[0]}x{m[1]}" == k))
                               for k in sorted({f"{m[0]}x{m[1]}" for m in meta})},
            "value": frames / (ms_t / 1e3), "unit": "frames/s", "ms_per_run": ms_t,
            "graph_launches_per_run": 1, "kernel_launches_per_run": launches // steps,
            "cycles": st_t["cycles"], "linesearch_rounds": st_t["linesearch_rounds"],
            "iterations": {"min": int(iters.min()), "max": int(iters.max()), "mean": float(iters.mean())},
            "default_schedule": {"value": frames / (ms_d / 1e3), "ms_per_run": ms_d},
            "host_launched_cycles": {"value": frames / (ms_h / 1e3), "ms_per_run": ms_h, "cycles": st_h["cycles"]},
            "one_batch_per_group": {"value": fr1 / (ms1 / 1e3), "groups": n1, "frames": fr1},
            "graph_equals_host_cycles": bool(same), "max_px_diff_tuned_vs_default_schedule": sched_diff,
            "autotune": {"seconds": tune_s, "choices": choices, "median_ms": timings,
                         "validation": tuner.last_validation},
            "fp64_path": {"value": frames / (ms_64 / 1e3), "ms_per_run": ms_64},
            "error_vs_fp64": err}


# ------------------------------------------------------------------------------------------------
# clocks during the timed region

class ClockSampler:
    QUERY = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap,power.draw")

    def __init__(self, index=0):
        self.rows, self.proc, self.index = [], None, index

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 8:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if r[3 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_summary():
    p = os.path.join(ROOT, "profiles", "k_trial_round_traffic.json")
    if os.path.exists(p):
        return json.load(open(p))
    return None


# ------------------------------------------------------------------------------------------------

def pipeline(groups, dev_frames, results, settings, lay, device, recon_frames: int, cpu: bool = True) -> dict:
    """The rows either side of the alignment on the same workload: the reference driver's frame
    preparation (ss_prepare_frames: block reorder of raw frames, and with the prefilter
    pregauss = 1, mednorm) over all frames, and the reconstruction (ss_reconstruct_frames) of one
    set of ``recon_frames`` frames of the first group with the knots this run estimated."""
    import torch

    from steadyscan_b200 import api, prep
    gidx = torch.from_numpy(np.asfortranarray(prep._block_gather_index(lay.prevknotind, lay.frame_w))
                            .reshape(-1, order="F")).to(device)
    valid = gidx >= 0
    h, w = lay.prevknotind.shape
    per = lay.frame_h * lay.frame_w
    # raw frames (h x w column-major each) from the block frames: the inverse of the block map
    flat = torch.cat(dev_frames)
    n = flat.numel() // per
    bm = flat.view(torch.int16).view(n, per)  # same bits; index_put has no uint16 kernel
    raw16 = torch.zeros((n, h * w), dtype=torch.int16, device=device)
    raw16[:, gidx[valid]] = bm[:, valid]
    raw3 = raw16.view(torch.uint16).view(n, w, h).permute(2, 1, 0)  # h x w x n, column-major per frame
    out = {}
    for name, kw in (("block_reorder_u16", dict(out_dtype=np.uint16)),
                     ("prefilter_f64", dict(pregauss=1.0, mednorm=True, out_dtype=np.float64))):
        for _ in range(3):  # warm-up: work memory and the output's first allocation
            api.prepare_frames(raw3, lay, **kw)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        got = api.prepare_frames(raw3, lay, **kw)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        # algorithmic bytes: the raw frames read once and the block matrices written once
        ob = 2 if name == "block_reorder_u16" else 8
        algo = n * (h * w * 2 + lay.frame_h * lay.frame_w * ob)
        pk, pk_kind = peaks()
        out[name] = {"frames": n, "frames_per_s": n / dt, "ms": dt * 1e3,
                     "roofline": {"bound": "hbm", "algorithmic_bytes": algo, "achieved_gbs": algo / dt / 1e9,
                                  "frac": algo / dt / 1e9 / pk, "peak": pk, "peak_source": pk_kind,
                                  "note": "whole call timed on the host (work memory, launches and the "
                                          "blur's and median's extra passes included)"}}
        if name == "block_reorder_u16":
            out[name]["equals_block_frames"] = bool(torch.equal(got.T.reshape(-1).view(torch.int16),
                                                                flat.view(torch.int16)))
    g0, r0 = groups[0], results[0]
    k = min(recon_frames, int(g0["nFrames"]))
    nk = lay.frame_w + 1
    dxk = np.asarray(r0["dx"]).reshape(nk, -1, order="F")[:, :k]
    dyk = np.asarray(r0["dy"]).reshape(nk, -1, order="F")[:, :k]
    fr = (raw16[:k].to(torch.int32) & 0xFFFF).to(torch.float32).view(k, w, h).permute(2, 1, 0)
    th, tw = np.asarray(g0["template_image"]).shape
    api.reconstruct_frames(fr[:, :, :2], dxk[:, :2], dyk[:, :2], settings, (th, tw))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rc = api.reconstruct_frames(fr, dxk, dyk, settings, (th, tw))
    dt = time.perf_counter() - t0
    out["reconstruct"] = {"frames": k, "frames_per_s": k / dt, "ms": dt * 1e3,
                          "sweeps_mean": float(np.mean(rc["iterations"])),
                          "masked_fraction": float(rc["mask"].mean()),
                          "note": "one set (one invert_bilinear_sampling call) of the first group's frames, "
                                  "template 512x512, ibs_regfac 3e-3, host output"}
    if cpu:
        # CPU baselines: the numpy restatements of the reference's MATLAB code on a bounded sample
        # (one host thread: numpy's FFT and scipy's sparse products are single-threaded)
        from oracle import frontend as ofe
        from oracle import reconstruct as orc
        nfc, nrc = 16, 4
        host = raw16[:nfc].cpu().numpy().view(np.uint16).reshape(nfc, w, h).transpose(2, 1, 0)
        for name, gsd, med in (("block_reorder_u16", 0.0, False), ("prefilter_f64", 1.0, True)):
            t0 = time.perf_counter()
            ofe.set_bmdata(host, lay.prevknotind, lay.frame_w, lay.cropping, gsd, med)
            dtc = time.perf_counter() - t0
            out[name]["cpu_baseline"] = {"frames_per_s": nfc / dtc, "cores": 1, "kind": "port",
                                         "sample": f"{nfc} frames, numpy restatement (FFT blur)"}
        t0 = time.perf_counter()
        orc.invert_bilinear_sampling(host[:, :, :nrc].astype(np.float32), dxk[:, :nrc], dyk[:, :nrc],
                                     settings["basex"], settings["basey"], settings["tfrac"],
                                     settings["prevknotind"], th, tw)
        dtc = time.perf_counter() - t0
        out["reconstruct"]["cpu_baseline"] = {"frames_per_s": nrc / dtc, "cores": 1, "kind": "port",
                                              "sample": f"the set's first {nrc} frames, numpy/scipy restatement"}
    return out


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The slowest rank's time (every rank calls this at the same point)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_sample(groups, n_frames, threads):
    """The FP64 CPU restatement on the first ``n_frames`` frames of the first group (frames/s)."""
    from oracle import oracle
    oracle.build()
    a = dict(groups[0])
    hb, w = a["tfrac"].shape
    a["bmData"] = np.asarray(a["bmData"])[:, :w * n_frames].astype(np.float64)
    a["nFrames"] = n_frames
    a["est_dx_knots"] = np.zeros((w + 1, n_frames))
    a["est_dy_knots"] = np.zeros((w + 1, n_frames))
    a["flags"] = "D"
    t0 = time.perf_counter()
    o = oracle.align_group(a, n_threads=threads, want_mask=False)
    dt = time.perf_counter() - t0
    return n_frames / dt, dt, o, a


def plain_path(groups, precision, n_groups):
    """The unbatched per-group path: one synchronous align_group_to_template call per group from host
    memory, one group after another, as the reference's caller drives it (frames/s)."""
    from steadyscan_b200 import api
    gs = []
    for g in groups[:max(1, n_groups)]:
        d = dict(g)
        d["flags"] = precision
        gs.append(d)
    for d in gs[:3]:  # warm-up
        api.align_group(d, want_mask=False)
    t0 = time.perf_counter()
    frames = 0
    for d in gs:
        api.align_group(d, want_mask=False)
        frames += int(d["nFrames"])
    return frames / (time.perf_counter() - t0), frames


def precision_sweep(a, o, template_shape):
    """Storage choices of precision S on the oracle's sample: frames uint16 / FP16 x template and
    gradients FP32 / FP16, each against the FP64 oracle: RMS and max knot error (px) and the relative
    L2 of the corrected frames."""
    from steadyscan_b200 import api, correct
    n = int(a["nFrames"])
    geo = (a["tfrac"], a["basex"], a["basey"], a["base_mask"])
    ref_c, ref_w = correct.correct_frames(a["bmData"], o["dx"], o["dy"], *geo, n, template_shape)
    counts = np.rint(np.asarray(a["bmData"])).astype(np.uint16)
    out = []
    for fname, fr in (("uint16", counts), ("float16", counts.astype(np.float16))):
        for tname in ("f32", "f16"):
            b = dict(a)
            b["bmData"] = np.asfortranarray(fr)
            b["flags"] = "S"
            g = api.align_group(b, want_mask=False, template_storage=tname)
            d = np.concatenate([g["dx"] - o["dx"], g["dy"] - o["dy"]])
            c, w = correct.correct_frames(a["bmData"], g["dx"], g["dy"], *geo, n, template_shape)
            out.append({"frames": fname, "template": tname, "rms_px": float(np.sqrt(np.mean(d * d))),
                        "max_px": float(np.max(np.abs(d))),
                        "corrected_rel_l2": correct.relative_l2(c, w, ref_c, ref_w)})
    # control: the FP64 path on the template rounded to FP16 separates the storage path's error
    # from the quantisation of the template itself
    from steadyscan_b200 import prep
    t16 = np.asarray(a["template_image"]).astype(np.float16).astype(np.float64)
    b = dict(a)
    b["bmData"] = np.asfortranarray(counts)
    b["flags"] = "D"
    b["template_image"] = t16
    b["xgrad"], b["ygrad"] = prep.template_gradients(t16)
    g = api.align_group(b, want_mask=False)
    d = np.concatenate([g["dx"] - o["dx"], g["dy"] - o["dy"]])
    c, w = correct.correct_frames(a["bmData"], g["dx"], g["dy"], *geo, n, template_shape)
    out.append({"frames": "uint16", "template": "f16-rounded, FP64 path (control)",
                "rms_px": float(np.sqrt(np.mean(d * d))), "max_px": float(np.max(np.abs(d))),
                "corrected_rel_l2": correct.relative_l2(c, w, ref_c, ref_w)})
    return {"sample": f"{n} frames of one 512x512 group vs the FP64 oracle", "variants": out}


def storage_sweep(args, device) -> dict:
    """The storage choices on the full 4000-frame workload of 512x512 frames with knots every 2 lines
    (the headline generator, seed 1004): frames uint16 / FP16 x template and gradients FP32 / FP16 in
    precision S, each one batch timed on device-resident frames, and each against the precision-D
    (FP64) run of the same batch: RMS and max knot difference (px) and the fraction of knots within
    0.05 px. A control runs precision D on the template rounded to FP16."""
    import torch

    from steadyscan_b200 import api, prep
    from steadyscan_b200._lib import SS_F16, SS_U16
    n = args.sweep_frames
    groups, dev, _, lay = make_workload(n, 512, 64, "S", 1004, device)
    f16 = [(t.view(torch.int16).to(torch.int32) & 0xFFFF).to(torch.float16) for t in dev]
    torch.cuda.synchronize()

    def run(frames, dtype, flags, tstore=None, template=None):
        grads = prep.template_gradients(template) if template is not None else None
        gs = []
        for g, t in zip(groups, frames):
            d = dict(g)
            d["bmData"] = api.DeviceMatrix(t.data_ptr(), lay.frame_h, lay.frame_w * int(g["nFrames"]), dtype, owner=t)
            d["flags"] = flags
            if template is not None:
                d["template_image"] = template
                d["xgrad"], d["ygrad"] = grads
            gs.append(d)
        b = api.Batch(gs, template_storage=tstore)
        b.run()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        b.run()
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        r = b.collect()
        b.close()
        # frames the reference's caller marks failed (steady_scan.m:246-284): correlation below
        # corr_thresh 0.75, or fewer than minblockfrac 0.25 of the blocks with a valid pixel
        ok = np.concatenate([(x["frame_corr"] >= 0.75) & (x["blocks_used"].mean(axis=0) >= 0.25) for x in r])
        return (np.concatenate([x["dx"] for x in r]), np.concatenate([x["dy"] for x in r]), ok), n / dt

    def err(k, ref):
        d = np.concatenate([k[0] - ref[0], k[1] - ref[1]])
        keep = np.repeat(ref[2], lay.frame_w + 1)  # the knots of the frames the caller keeps (D run)
        da = np.concatenate([(k[0] - ref[0])[keep], (k[1] - ref[1])[keep]])
        return {"rms_px": float(np.sqrt(np.mean(d * d))), "max_px": float(np.max(np.abs(d))),
                "within_0p05_px": float(np.mean(np.abs(d) <= 0.05)),
                "accepted_frames": int(ref[2].sum()), "rms_px_accepted": float(np.sqrt(np.mean(da * da))),
                "max_px_accepted": float(np.max(np.abs(da)))}

    ref, v_d = run(dev, SS_U16, "D")
    out = {"workload": f"{n} frames of 512x512, knots every 2 lines, groups of 64, lambda 5e-3; "
                       "accuracy against the precision-D (FP64) run of the same frames",
           "D_frames_per_s": v_d, "variants": []}
    for fname, frames, dt in (("uint16", dev, SS_U16), ("float16", f16, SS_F16)):
        for tname in ("f32", "f16"):
            k, v = run(frames, dt, "S", tname)
            out["variants"].append(dict(frames=fname, template=tname, frames_per_s=v, **err(k, ref)))
    t16 = np.asarray(groups[0]["template_image"]).astype(np.float16).astype(np.float64)
    k, v = run(dev, SS_U16, "D", template=t16)
    out["control_fp64_on_f16_rounded_template"] = dict(frames_per_s=v, **err(k, ref))
    return out


def serve(args, device, seconds, plain_d):
    """Serving load: 8 sessions, each with its own 512x512 template; groups of 1-64 frames arrive
    per session as a Poisson process at 30 Hz, doubled for 2 s of every 10 s. Frames come from a
    per-session pool rendered on the GPU; each session's later groups start from its last knots."""
    import torch
    from steadyscan_b200 import api, serving
    from steadyscan_b200._lib import SS_U16
    n_ses, pool_frames = 8, 512
    server = serving.Server(memory_budget=24 << 30, device=device.index or 0, max_active=96,
                            warm_start=args.serve_warm)
    pools = []
    for s in range(n_ses):
        groups, dev, _, lay = make_workload(pool_frames, 512, pool_frames, "S", 1005 + 31 * s, device)
        server.add_session(groups[0])
        pools.append((dev[0], lay))
    torch.cuda.synchronize()
    rng = np.random.default_rng(1005)
    sched = serving.arrival_schedule(n_ses, seconds, 30.0, 10.0, 2.0, 2.0, (1, 64), rng)
    cursor = [0] * n_ses
    t0 = time.perf_counter()
    k = 0
    while k < len(sched) or server.by_slot or server.pending:
        now = time.perf_counter() - t0
        while k < len(sched) and sched[k][0] <= now:
            t, s, n = sched[k]
            flat, lay = pools[s]
            if cursor[s] + n > pool_frames:
                cursor[s] = 0
            f0 = cursor[s]
            cursor[s] += n
            px = lay.frame_h * lay.frame_w
            view = flat[f0 * px:(f0 + n) * px]
            m = api.DeviceMatrix(view.data_ptr(), lay.frame_h, lay.frame_w * n, SS_U16, owner=view)
            r = server.submit(s, m, n, t_arrival=t0 + t)
            r.in_burst = (t % 10.0) < 2.0
            k += 1
        server.tick()
    elapsed = time.perf_counter() - t0
    st = serving.latency_stats(server.done)
    # the 2x bursts offer more frames than the server's capacity, so their groups queue; groups that
    # arrived outside the bursts show the latency of the steady load (queues left by a burst included)
    st_burst = serving.latency_stats([r for r in server.done if r.in_burst])
    st_steady = serving.latency_stats([r for r in server.done if not r.in_burst])
    offered = sum(n for _, _, n in sched) / seconds
    iters = [r.result["iter_used"] for r in server.done]
    out = {"sessions": n_ses, "seconds": seconds, "offered_frames_per_s": offered,
           "frames_per_s": st["frames"] / elapsed, "groups": st["groups"], "p50_ms": st["p50_ms"],
           "p99_ms": st["p99_ms"], "max_ms": st["max_ms"],
           "outside_bursts": {k: st_steady[k] for k in ("groups", "p50_ms", "p99_ms", "max_ms")},
           "inside_bursts": {k: st_burst[k] for k in ("groups", "p50_ms", "p99_ms", "max_ms")},
           "admission": "first come, first served in arrival order, while the device memory budget has room",
           "peak_in_flight": server.peak_active,
           "peak_device_bytes": server.peak_bytes, "server_cycles": server.cycles,
           "ms_per_cycle": 1000.0 * elapsed / max(1, server.cycles),
           "iterations_mean": float(np.mean(iters)) if iters else None,
           "plain_serial_frames_per_s": plain_d,
           "warm_start": args.serve_warm,
           "load": "Poisson 30 Hz per session, 2x for 2 s of every 10 s, groups U[1,64] frames of 512x512 uint16, "
                   "precision S"}
    server.close()
    return out


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    threads = os.cpu_count() or 1

    if args.impl == "reference":
        if rank != 0:
            return
        groups, _, _, _ = make_workload_cpu(args)
        vals = []
        for i in range(args.warmup + args.steps):
            v, dt, _, _ = cpu_sample(groups, args.cpu_sample_frames, threads)
            if i >= args.warmup:
                vals.append(v)
        value = float(np.mean(vals))
        sample = f"{args.cpu_sample_frames} frames of one {args.size}x{args.size} group, FP64, {threads} threads"
        print(json.dumps({"impl": "reference", "metric": METRIC, "value": value, "unit": "frames/s",
                          "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": 1000.0 * args.cpu_sample_frames / value, "higher_is_better": True,
                          "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                          "config": workload_config(args),
                          "cpu_baseline": {"value": value, "unit": "frames/s", "cores": threads, "kind": "port",
                                           "sample": sample},
                          "e2e": {"value": value, "unit": "frames/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}))
        return

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    device = torch.device("cuda", local)
    from steadyscan_b200 import api
    from steadyscan_b200._lib import SS_U16

    if args.only_ragged:
        if rank == 0:
            print(json.dumps({"ragged": ragged(args, device)}))
        return

    groups, dev_frames, settings, lay = make_workload(args.frames, args.size, args.group, args.precision,
                                                      1002 + 17 * rank, device)
    torch.cuda.synchronize()
    # device-resident inputs for `value`
    dgroups = []
    for g, t in zip(groups, dev_frames):
        d = dict(g)
        d["bmData"] = api.DeviceMatrix(t.data_ptr(), lay.frame_h, lay.frame_w * int(g["nFrames"]), SS_U16, owner=t)
        dgroups.append(d)
    batch = api.Batch(dgroups)
    stream = torch.cuda.ExternalStream(batch.stream_ptr, device=device)

    if args.only_pipeline:  # the rows either side of the alignment, on this workload's frames and knots
        batch.run()
        results = batch.collect()
        batch.close()
        if rank == 0:
            print(json.dumps({"pipeline": pipeline(groups, dev_frames, results, settings, lay, device,
                                                   args.recon_frames, cpu=not args.no_cpu)}))
        return

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        batch.run()
    barrier()
    launches = 0
    with ClockSampler(local) as clk:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            batch.run()
            launches += batch.stats()["kernel_launches"]
        e1.record(stream)
        barrier()
    ms_total = max_over_ranks(e0.elapsed_time(e1), dist, device)
    ms_step = ms_total / args.steps
    value = args.frames * world / (ms_step / 1000.0)
    st = batch.stats()

    # roofline of the evaluation kernel from one extra run with event timing inside the engine
    batch.set_timing(True)
    batch.run()
    torch.cuda.synchronize()
    rs = batch.stats()
    batch.set_timing(False)
    results = batch.collect()
    frame_bytes = lay.frame_h * lay.frame_w * 2
    passes = rs["frame_passes"]
    ems = rs["eval_ms"]
    peak, peak_kind = peaks()
    tr = traffic_summary()
    # the dominant kernel: the line-search trial rounds; one frame-trial reads one frame
    n_launch = max(1, rs["linesearch_rounds"])
    units = passes[1] / n_launch
    launch_ms = ems[1] / n_launch
    achieved = units * frame_bytes / (launch_ms / 1e3) / 1e9 if launch_ms > 0 else None
    by_pass = {}
    # assembly columns whose knots had not moved kept their sums and read no frame data
    kept_frames = rs["assembly_columns_kept"] / lay.frame_w
    for i, name in enumerate(("assembly", "trial", "correlation", "final")):
        reads = passes[i] - (kept_frames if i == 0 else 0)
        gbs = reads * frame_bytes / (ems[i] / 1e3) / 1e9 if ems[i] > 0 else None
        by_pass[name] = {"frame_passes": passes[i], "frame_reads": reads, "ms": ems[i], "achieved_gbs": gbs,
                         "frac": gbs / peak if gbs else None}
    by_pass["frame_reads_per_evaluation"] = (sum(passes) - kept_frames) / max(1, sum(r["n_frame_passes"]
                                                                                  for r in results))
    roofline = {"kernel": "k_trial_round (line-search trial rounds, the largest share of device time)",
                "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
                "traffic": tr["bytes_per_frame_pass"] * units if tr else None,
                "algorithmic_bytes_per_launch": units * frame_bytes, "launch_ms": launch_ms,
                "launches": n_launch, "by_pass": by_pass,
                "eval_share_of_step": sum(ems) / rs["run_ms"] if rs["run_ms"] else None,
                "staging": rs["staging"]}

    # end to end through the public C ABI from pinned host memory
    e2e = None
    if not args.no_e2e:
        pinned = []
        hgroups = []
        h2d = 0
        shared_seen = set()
        # ss_align_groups runs host-resident groups as one batch, which uploads each buffer the groups
        # share once
        for gi, g in enumerate(groups):
            d = dict(g)
            src = np.asarray(g["bmData"])
            pt = torch.empty(src.size, dtype=torch.int16, pin_memory=True)
            pv = pt.numpy().view(np.uint16).reshape(src.shape, order="F")
            pv[...] = src
            pinned.append(pt)
            d["bmData"] = pv
            hgroups.append(d)
            h2d += src.nbytes + 16 * (lay.frame_w + 1) * int(g["nFrames"])  # frames + initial knots
            for k in ("template_image", "xgrad", "ygrad", "tfrac", "basex", "basey", "base_mask"):
                if id(g[k]) not in shared_seen:  # one upload per distinct buffer
                    shared_seen.add(id(g[k]))
                    h2d += np.asarray(g[k]).nbytes
        api.align_groups(hgroups, want_mask=False)  # warm-up
        barrier()
        t0 = time.perf_counter()
        for _ in range(max(1, args.steps)):
            res = api.align_groups(hgroups, want_mask=False)
        torch.cuda.synchronize()
        dt = max_over_ranks((time.perf_counter() - t0) / max(1, args.steps), dist, device)
        w1 = lay.frame_w + 1
        d2h = sum(int(g["nFrames"]) * (2 * w1 + 2) * 8 + 8 for g in groups)
        e2e = {"value": args.frames * world / dt, "unit": "frames/s", "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "api": "ss_align_groups"}

    plain = None
    if rank == 0 and not args.no_plain:
        plain = {}
        for prec in ("D", "S"):
            v, nfr = plain_path(groups, prec, args.plain_groups)
            plain[prec] = {"value": v, "unit": "frames/s", "frames": nfr}
        plain["path"] = ("unbatched: one synchronous ss_align_group_to_template call per group of "
                         f"{args.group} frames from host memory, serially")
        plain["batched_vs_plain_D"] = value / plain["D"]["value"]
        if e2e:
            plain["e2e_vs_plain_D"] = e2e["value"] / plain["D"]["value"]

    cpu = None
    acc = None
    if rank == 0 and not args.no_cpu:
        v, dt, o, a = cpu_sample(groups, args.cpu_sample_frames, threads)
        cpu = {"value": v, "unit": "frames/s", "cores": threads, "kind": "port",
               "sample": f"{args.cpu_sample_frames} frames of one {args.size}x{args.size} group, FP64 oracle, "
                         f"{dt:.1f} s"}
        if args.cpu_single_frames > 0:
            v1, dt1, _, _ = cpu_sample(groups, args.cpu_single_frames, 1)
            cpu["single_thread"] = {"value": v1, "unit": "frames/s", "cores": 1,
                                    "sample": f"the first {args.cpu_single_frames} frames of the same group, "
                                              f"{dt1:.1f} s"}
        # accuracy of the timed precision against the FP64 oracle on that sample
        a2 = dict(a)
        a2["flags"] = args.precision
        g = api.align_group(a2, want_mask=False)
        rms = float(np.sqrt(np.mean(np.concatenate([g["dx"] - o["dx"], g["dy"] - o["dy"]]) ** 2)))
        mx = float(np.max(np.abs(np.concatenate([g["dx"] - o["dx"], g["dy"] - o["dy"]]))))
        acc = {"rms_px_vs_fp64": rms, "max_px_vs_fp64": mx, "sample": f"{args.cpu_sample_frames} frames"}
        if not args.no_sweep:
            acc["precision_sweep"] = precision_sweep(a, o, np.asarray(a["template_image"]).shape)

    small_line = None
    if rank == 0 and not args.no_cpu:
        small_line = plain_small(device, threads)

    ragged_line = None
    if rank == 0 and not args.no_ragged:
        ragged_line = ragged(args, device)

    sweep_line = None
    if rank == 0 and args.sweep_frames > 0:
        sweep_line = storage_sweep(args, device)

    pipeline_line = None
    if rank == 0 and not args.no_pipeline:
        pipeline_line = pipeline(groups, dev_frames, results, settings, lay, device, args.recon_frames,
                                 cpu=not args.no_cpu)

    serving_line = None
    if rank == 0 and args.serve_seconds > 0:
        batch.close()
        serving_line = serve(args, device, args.serve_seconds, plain["D"]["value"] if plain else None)

    if rank == 0:
        iters = [r["iter_used"] for r in results]
        line = {"metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32" if args.precision == "S" else "f64", "data": "synthetic",
                "config": workload_config(args), "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e,
                "clocks": clk.summary(), "gpu_launches": launches, "accuracy": acc, "plain_gpu": plain,
                "plain_method_small": small_line, "ragged": ragged_line, "serving": serving_line,
                "pipeline": pipeline_line, "storage_sweep": sweep_line,
                "run": {"cycles": st["cycles"], "linesearch_rounds": st["linesearch_rounds"],
                        "iterations_min": int(min(iters)), "iterations_max": int(max(iters)),
                        "arena_bytes": st["arena_bytes"]}}
        print(json.dumps(line))
    batch.close()
    if dist:
        dist.destroy_process_group()


def workload_config(args):
    return {"workload": f"{args.frames} frames {args.size}x{args.size} uint16, knots every 2 lines "
                        f"({args.size // 2 + 1} knots), groups of {args.group} frames, precision {args.precision} "
                        f"(FP32 pixel arithmetic, FP64 reduction and solve), lambda 5e-3, default settings",
            "frames": args.frames, "group_frames": args.group, "frame_size": args.size,
            "l2": "frames resident in HBM exceed L2 (1 GB vs 126 MB); no flush"}


def make_workload_cpu(args):
    import torch
    return make_workload(min(args.frames, args.cpu_sample_frames), args.size, args.group, "D", 1002, "cpu")


if __name__ == "__main__":
    main()
