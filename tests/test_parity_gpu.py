"""Parity of the CUDA path (through the C ABI) with the FP64 oracle on identical inputs.

Precision 'D' follows the reference's FP64 arithmetic; its sums are reduced in a different order
than the oracle's sequential loops, so knots agree to ~1e-9 px rather than bit for bit. Masks and
iteration counts are compared exactly. Precision 'S' (FP32 pixel arithmetic, FP64 reduction and
solve) is held to the 0.02 px RMS bound on displacements.
"""
import numpy as np
import pytest

from oracle import oracle
from steadyscan_b200 import api
from tests.helpers import knot_rms, make_args

pytestmark = pytest.mark.gpu

KNOT_TOL_D = 1e-6     # px, precision 'D'
KNOT_RMS_S = 0.02     # px RMS, precision 'S'


def _compare_d(args, o=None, g=None, check_mask=True):
    o = o or oracle.align_group(args)
    g = g or api.align_group(args)
    assert g["iter_used"] == o["iterations"], (g["iter_used"], o["iterations"])
    assert g["stop_reason"] == o["stop_reason"]
    np.testing.assert_allclose(g["dx"], o["dx"], atol=KNOT_TOL_D, rtol=0)
    np.testing.assert_allclose(g["dy"], o["dy"], atol=KNOT_TOL_D, rtol=0)
    np.testing.assert_allclose(g["frame_corr"], o["frame_corr"], atol=1e-9, rtol=1e-9, equal_nan=True)
    np.testing.assert_allclose(g["residrms"], o["residrms"], rtol=1e-9, atol=1e-9, equal_nan=True)
    if check_mask:
        np.testing.assert_array_equal(g["mask"], o["mask"])
    return o, g


CASES = {
    "even_default": dict(),
    "odd_frames": dict(n_frames=3),
    "one_frame_groupsize1": dict(n_frames=1, settings={"gpu_frame_groupsize": 1}),
    "nonint_lines_per_knot": dict(nlines=30, linewidth=20, nknots=8),
    "bidirectional_k1": dict(nlines=16, linewidth=16, nknots=17, settings={"isbidirectional": True}),
    "solver1_nofilter": dict(settings={"gpu_solver_id": 1, "gpu_filter_id": 0}),
    "range_filter": dict(settings={"gpu_filter_id": 2}),
    "ilu_solver0": dict(settings={"gpu_solver_id": 0}),
    # 3-tap median of the solved step before the line search (flag R; d_medianfilter.cu:3-20)
    "median_before_linesearch": dict(settings={"gpu_flags": "R"}, seed=15),
    "median_before_linesearch_solver1": dict(settings={"gpu_flags": "R", "gpu_solver_id": 1, "gpu_filter_id": 0},
                                             n_frames=6, seed=16),
    "big_motion": dict(clip_px=6.0, jumps=2, jump_px=4.0, seed=11),
    "template_larger": dict(template_size=(40, 44), seed=5),
    "uint16_frames": dict(frame_dtype=np.uint16, seed=8),
    # a knot chain longer than the solve's 1024 partitions: partitions with interior nodes
    "long_chain": dict(n_frames=72, nknots=17, seed=61),
    # huge first steps: trials with no block present whose moving knots are the frame's first
    "absent_trial_movement": dict(seed=45, n_frames=4, clip_px=6.0, jumps=2, jump_px=4.0,
                                  settings={"gpu_filter_max_iterations": 2}),
}


@pytest.mark.parametrize("name", list(CASES))
def test_precision_d_matches_oracle(name):
    kw = dict(CASES[name])
    args, _, _ = make_args(**kw)
    _compare_d(args)


@pytest.mark.parametrize("solver", [0, 2])
def test_lambda_regulariser(solver):
    args, _, _ = make_args(seed=21)
    args["lambda"] = 50.0
    args["solver_id"] = solver
    _compare_d(args)


@pytest.mark.parametrize("flags", ["D", "S"])
def test_assembly_keeps_columns_with_unchanged_knots(flags):
    """Block columns whose knots did not move since their last assembly keep its sums instead of
    reading the frame again; the run still matches the oracle (D) or the bound (S). In this case
    frames stand still for whole iterations (their knots equal across the oracle's knot history)."""
    args, _, _ = make_args(n_frames=16, seed=23, frame_dtype=np.uint16)
    o = oracle.align_group(args)
    b = api.Batch([dict(args, flags=flags)], want_mask=True)
    b.run()
    g = b.collect()[0]
    st = b.stats()
    b.close()
    assert st["assembly_columns_kept"] > 0
    if flags == "D":
        _compare_d(args, o=o, g=g)
    else:
        assert knot_rms(np.concatenate([g["dx"], g["dy"]]), np.concatenate([o["dx"], o["dy"]])) <= KNOT_RMS_S


def test_ilu_solver0_long_chain_and_precision_s():
    """ILU(0) (solver id 0) over a chain longer than the exact solve's partitions, in precision D
    against the oracle, and in precision S within the bound."""
    args, _, _ = make_args(n_frames=24, nknots=17, seed=62, settings={"gpu_solver_id": 0}, frame_dtype=np.uint16)
    o, _ = _compare_d(args)
    g = api.align_group(dict(args, flags="S"))
    assert knot_rms(np.concatenate([g["dx"], g["dy"]]), np.concatenate([o["dx"], o["dy"]])) <= KNOT_RMS_S


def test_flags_history_outputs():
    args, _, _ = make_args(seed=4)
    args["flags"] = "DCcePp"
    o = oracle.align_group(args, want_history=True)
    g = api.align_group(args, want_history=True)
    it = o["iterations"]
    assert g["iter_used"] == it
    np.testing.assert_allclose(g["iteration_corr"][:it], o["iter_corr"][:it], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(g["frame_corr_history"][:, :it], o["frame_corr_hist"][:it].T, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(g["all_params"][:, :it], o["all_params"][:it].T, atol=KNOT_TOL_D)
    # frame-ordered parameters (flag p): nF x 2(W+1), x knots then y knots
    w1 = args["tfrac"].shape[1] + 1
    fp = g["frame_params"]
    np.testing.assert_allclose(fp[:, :w1].reshape(-1), o["dx"].reshape(-1, w1).reshape(-1), atol=KNOT_TOL_D)
    np.testing.assert_allclose(fp[:, w1:].reshape(-1), o["dy"].reshape(-1, w1).reshape(-1), atol=KNOT_TOL_D)
    np.testing.assert_allclose(g["raw_params"], o["p_last"], atol=KNOT_TOL_D)


def test_mask_inactive_flag():
    args, _, _ = make_args(n_frames=4, seed=6)
    args["flags"] = "DMc"
    args["halt_correlation"] = 0.9
    _compare_d(args)


def _compare_history(args):
    o, g = _compare_d(args, o=oracle.align_group(args, want_history=True), g=api.align_group(args, want_history=True))
    it = o["iterations"]
    np.testing.assert_allclose(g["iteration_corr"][:it], o["iter_corr"][:it], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(g["frame_corr_history"][:, :it], o["frame_corr_hist"][:it].T, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(g["all_params"][:, :it], o["all_params"][:it].T, atol=KNOT_TOL_D)
    return o, g


# Flag t (TimedMainIteration): the cases of the timed reference-run fixtures
TIMED = {
    "retry_odd": dict(n_frames=3, seed=6, settings={"gpu_solver_id": 1}),
    "filter_limit": dict(seed=41, n_frames=4, clip_px=6.0, jumps=2, jump_px=4.0,
                         settings={"gpu_solver_id": 1, "gpu_filter_max_iterations": 2}),
    "mask_inactive": dict(n_frames=6, seed=10, settings={"gpu_solver_id": 1, "haltcorr": 0.15}),
}


@pytest.mark.parametrize("name", list(TIMED))
def test_flag_t_timed_iteration_and_rg_params(name):
    """Flag t switches to TimedMainIteration's bookkeeping (paramsUsed cleared every half-step,
    its filterID rules, the retry as the next iteration) and fills output 14 with the chain after
    every half-step."""
    args, _, _ = make_args(**TIMED[name])
    args["flags"] = "DCcet" + ("M" if name == "mask_inactive" else "")
    o, g = _compare_history(args)
    k = 2 * o["iterations"] + 2
    rg = g["rg_params"]
    assert rg.shape == (2 * (args["tfrac"].shape[1] * int(args["nFrames"]) + 1), 2 * int(args["max_iter"]))
    np.testing.assert_allclose(rg[:, :k], o["rg_params"][:k].T, atol=KNOT_TOL_D)
    assert not np.any(rg[:, k:])
    assert not np.any(g["function_times"][[0, 3, 6, 12, 13]])
    assert g["iteration_times"] is None  # output 9 needs flag T as well


def test_timing_outputs_flags_T_and_t():
    args, _, _ = make_args(seed=4, n_frames=6)
    g = api.align_group(dict(args, flags="STt"), want_history=True)
    it = g["iter_used"]
    ft, itt = g["function_times"], g["iteration_times"]
    assert ft.shape == (14,) and itt.shape == (int(args["max_iter"]),)
    assert np.all(ft[[1, 2, 4, 5, 7, 8, 9, 10, 11]] > 0) and not np.any(ft[[0, 3, 6, 12, 13]])
    assert ft.sum() <= g["elapsed_ms"] / 1000.0
    assert np.all(itt[:it] >= 0) and np.count_nonzero(itt[:it]) >= it - 1 and not np.any(itt[it:])
    assert itt.sum() <= g["elapsed_ms"] / 1000.0
    # the chain after the second half-step of every iteration is the iteration's chain (output 15),
    # one slot pair later when the iteration was retried without the filter
    rg, ap = g["rg_params"], g["all_params"]
    for j in range(it):
        assert any(np.array_equal(rg[:, s], ap[:, j]) for s in (2 * j + 1, 2 * j + 3) if s < rg.shape[1])
    g2 = api.align_group(dict(args, flags="ST"))
    assert not np.any(g2["function_times"]) and g2["iteration_times"] is None and g2["rg_params"] is None


@pytest.mark.parametrize("seed,halt", [(16, 0.2), (10, 0.15)])
def test_mask_inactive_frames_stale_over_iterations(seed, halt):
    """Flags M and c with frames inactive over consecutive iterations (the cases of the
    mask_inactive_stale reference-run fixtures): the difference-image buffer of an inactive frame is
    swapped by every global correlation past the swap-back index (task_correlation.cu:86-98) and
    read by the next assembly, correlation and final pass."""
    args, _, _ = make_args(n_frames=6, seed=seed, settings={"gpu_solver_id": 1, "haltcorr": halt})
    args["flags"] = "DCceM"
    o, _ = _compare_history(args)
    assert o["iterations"] >= 3


def test_frame_corr_past_the_swap_back_in_row_one():
    """Flag c on 40 frames of 8 blocks (fW = 320): the per-iteration frame correlations switch
    from the swapped image to the difference image at row-major index 512, inside row 1."""
    args, _, _ = make_args(n_frames=40, seed=33, settings={"gpu_solver_id": 1})
    args["flags"] = "DCce"
    _compare_history(args)
    args["flags"] = "SCce"
    o = oracle.align_group(dict(args, flags="DCce"), want_history=True)
    g = api.align_group(args, want_history=True)
    it = min(o["iterations"], g["iter_used"])
    np.testing.assert_allclose(g["frame_corr_history"][:, :it], o["frame_corr_hist"][:it].T, atol=2e-3)


def test_frames_outside_template():
    """Frames displaced entirely off the template: no block is ever present (steady_scan.m:267-272)."""
    args, _, _ = make_args(seed=9)
    args["est_dx_knots"] = np.full_like(args["est_dx_knots"], 500.0)
    o, g = _compare_d(args)
    assert not g["mask"].any()


def test_precision_s_within_bound():
    args, _, _ = make_args(frame_dtype=np.uint16, seed=12)
    o = oracle.align_group(args)
    args["flags"] = "S"
    g = api.align_group(args)
    assert knot_rms(np.concatenate([g["dx"], g["dy"]]), np.concatenate([o["dx"], o["dy"]])) <= KNOT_RMS_S


@pytest.mark.parametrize("dtype", [np.uint16, np.float16, np.float32, np.float64])
def test_precision_s_pixel_pairs_per_frame_type(dtype):
    """Precision S on the default scan geometry with 2 lines per knot (Hb a multiple of 64: the
    packed pixel-pair assembly) stays within the bound of the FP64 oracle on the same frames for
    every frame storage type; valid-pixel counts differ at most at boundary ties."""
    args, _, _ = make_args(nlines=64, linewidth=64, nknots=33, n_frames=4, seed=51, frame_dtype=dtype, n_blobs=30)
    o = oracle.align_group(args)
    args["flags"] = "S"
    g = api.align_group(args)
    assert knot_rms(np.concatenate([g["dx"], g["dy"]]), np.concatenate([o["dx"], o["dy"]])) <= KNOT_RMS_S
    assert abs(int(g["mask"].sum()) - int(o["mask"].sum())) <= 0.001 * g["mask"].size


def test_precision_s_affine_and_table_geometry_agree():
    """Precision S computes the default scan geometry in registers when the tables are affine; a
    1e-7 px perturbation of basex forces the table path. Both stay within the bound of FP64."""
    args, _, _ = make_args(frame_dtype=np.uint16, seed=13)
    o = oracle.align_group(args)
    args["flags"] = "S"
    g_aff = api.align_group(args)
    t = dict(args)
    t["basex"] = args["basex"] + 1e-7
    g_tab = api.align_group(t)
    ref = np.concatenate([o["dx"], o["dy"]])
    for g in (g_aff, g_tab):
        assert knot_rms(np.concatenate([g["dx"], g["dy"]]), ref) <= KNOT_RMS_S


@pytest.mark.parametrize("flags", ["D", "S"])
def test_batched_groups_sharing_template_and_geometry(flags):
    """Sets of one recording pass the same template and geometry arrays; the library converts and
    uploads them once and every set still gets its single-call result."""
    args, _, _ = make_args(n_frames=12, seed=41, frame_dtype=np.uint16)
    args["flags"] = flags
    w = args["tfrac"].shape[1]
    groups = []
    for k in range(3):
        a = dict(args)
        a["bmData"] = np.asfortranarray(args["bmData"][:, k * 4 * w:(k + 1) * 4 * w])
        a["nFrames"] = 4
        a["est_dx_knots"] = args["est_dx_knots"][:, k * 4:(k + 1) * 4]
        a["est_dy_knots"] = args["est_dy_knots"][:, k * 4:(k + 1) * 4]
        groups.append(a)
    batched = api.align_groups(groups)
    for a, b in zip(groups, batched):
        single = api.align_group(a)
        assert single["iter_used"] == b["iter_used"]
        np.testing.assert_array_equal(single["dx"], b["dx"])
        np.testing.assert_array_equal(single["dy"], b["dy"])
        np.testing.assert_array_equal(single["mask"], b["mask"])
    if flags == "D":
        _compare_d(groups[1], g=batched[1])


def test_batched_equals_single():
    """Ragged groups in one batched run give the same results as one call each."""
    specs = [dict(seed=31), dict(n_frames=3, seed=32), dict(nlines=24, linewidth=20, nknots=7, seed=33),
             dict(n_frames=6, seed=34, settings={"gpu_filter_id": 0})]
    groups = [make_args(**s)[0] for s in specs]
    batched = api.align_groups(groups)
    for a, b in zip(groups, batched):
        single = api.align_group(a)
        assert single["iter_used"] == b["iter_used"]
        np.testing.assert_array_equal(single["dx"], b["dx"])
        np.testing.assert_array_equal(single["dy"], b["dy"])
        np.testing.assert_array_equal(single["mask"], b["mask"])
        np.testing.assert_array_equal(single["residrms"], b["residrms"])


@pytest.mark.parametrize("prec", ["D", "S"])
def test_streamed_uploads_equal_the_resident_batch(prec):
    """ss_align_groups uploads host frames on a second stream while earlier groups run (each group
    joins when its frames have arrived): the results are those of a batch whose frames were all
    uploaded before the run."""
    specs = [dict(seed=41 + k, n_frames=2 + k % 3, frame_dtype=np.uint16) for k in range(6)]
    groups = [dict(make_args(**sp)[0], flags=prec) for sp in specs]
    streamed = api.align_groups(groups, want_mask=False)
    b = api.Batch(groups)
    b.run()
    resident = b.collect()
    b.close()
    for a, r in zip(streamed, resident):
        assert a["iter_used"] == r["iter_used"] and a["stop_reason"] == r["stop_reason"]
        for k in ("dx", "dy", "frame_corr", "residrms"):
            np.testing.assert_array_equal(a[k], r[k])


def test_concurrent_calls_share_the_staging_buffer():
    """Calls from several host threads at once (ctypes releases the GIL) take turns on the
    library's page-locked staging buffer for their small uploads and result copies: each call gets
    the results it gets alone."""
    import threading
    specs = [dict(seed=51 + k, n_frames=2 + k % 3, frame_dtype=np.uint16) for k in range(4)]
    groups = [dict(make_args(**sp)[0], flags="S" if k % 2 else "D") for k, sp in enumerate(specs)]
    alone = [api.align_group(g) for g in groups]
    out = [[] for _ in groups]
    errs = []

    def work(k):
        try:
            for _ in range(3):
                out[k].append(api.align_group(groups[k]))
        except Exception as e:  # noqa: BLE001 - reported below
            errs.append(e)

    threads = [threading.Thread(target=work, args=(k,)) for k in range(len(groups))]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not errs, errs
    assert not any(t.is_alive() for t in threads)
    for a, rs in zip(alone, out):
        assert len(rs) == 3
        for r in rs:
            assert a["iter_used"] == r["iter_used"]
            for k in ("dx", "dy", "frame_corr", "residrms", "mask"):
                np.testing.assert_array_equal(a[k], r[k])


def test_persistent_grid_many_tiles_precision_s():
    """A batch with more tiles (block column x frame chunk) than the persistent grid has CTAs, so
    every CTA takes several tiles, and searches spread over several cycles: each group still gets
    its single-call result."""
    groups = []
    for i in range(12):
        a, _, _ = make_args(nlines=64, linewidth=64, nknots=33, n_frames=40, seed=70 + i, n_blobs=30,
                            frame_dtype=np.uint16)
        a["flags"] = "S"
        groups.append(a)
    batched = api.align_groups(groups)
    for a, b in zip(groups, batched):
        single = api.align_group(a)
        assert single["iter_used"] == b["iter_used"]
        np.testing.assert_array_equal(single["dx"], b["dx"])
        np.testing.assert_array_equal(single["dy"], b["dy"])
        np.testing.assert_array_equal(single["mask"], b["mask"])


def test_fp16_template_storage_matches_fp64_on_the_rounded_template():
    """Template and gradients stored in FP16 (precision S): the error against FP64 comes from rounding
    the template itself, so the storage path agrees with the FP64 path run on the FP16-rounded
    template within the precision-S bound."""
    from steadyscan_b200 import prep
    args, _, _ = make_args(frame_dtype=np.uint16, seed=14)
    t16 = np.asarray(args["template_image"]).astype(np.float16).astype(np.float64)
    d = dict(args)
    d["template_image"] = t16
    d["xgrad"], d["ygrad"] = prep.template_gradients(t16)
    ref = api.align_group(d)
    s = dict(args)
    s["flags"] = "S"
    g = api.align_group(s, template_storage="f16")
    assert knot_rms(np.concatenate([g["dx"], g["dy"]]), np.concatenate([ref["dx"], ref["dy"]])) <= KNOT_RMS_S


@pytest.mark.parametrize("flags", ["D", "S"])
def test_graph_run_equals_host_launched_cycles(flags):
    """The run as one CUDA graph (device-side loops over cycles and trial rounds) gives every group
    of a ragged batch the result of host-launched cycles, bit for bit."""
    specs = [dict(seed=81, frame_dtype=np.uint16), dict(n_frames=3, seed=82, frame_dtype=np.uint16),
             dict(nlines=24, linewidth=20, nknots=7, seed=83, frame_dtype=np.uint16),
             dict(nlines=64, linewidth=64, nknots=33, n_frames=9, seed=84, n_blobs=30, frame_dtype=np.uint16)]
    groups = []
    for s in specs:
        a = make_args(**s)[0]
        a["flags"] = flags
        groups.append(a)
    res = []
    for graph in (True, False):
        b = api.Batch(groups, want_mask=True)
        b.set_graph(graph)
        b.run()
        res.append((b.collect(), b.stats()))
    (rg, sg), (rh, sh) = res
    for a, b in zip(rg, rh):
        assert a["iter_used"] == b["iter_used"]
        np.testing.assert_array_equal(a["dx"], b["dx"])
        np.testing.assert_array_equal(a["dy"], b["dy"])
        np.testing.assert_array_equal(a["mask"], b["mask"])
        np.testing.assert_array_equal(a["residrms"], b["residrms"])
    assert sg["cycles"] > 0 and sg["kernel_launches"] > 0
    assert sg["cycles"] <= sh["cycles"]
