"""Host logic of bench.py on CPU: the reference arm end to end on a tiny workload, and the
max-over-ranks timing reduction across two gloo ranks (the N > 1 path)."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_prints_one_json_line():
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--size", "32", "--frames", "4",
           "--cpu-sample-frames", "2", "--steps", "1", "--warmup", "1"]
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "frames/s" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["e2e"]["h2d_bytes_per_step"] == 0


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    v = bench.max_over_ranks(10.0 + rank * 5.0, dist, "cpu")
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, v))


def test_max_over_ranks_gloo_two_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = dict(q.get(timeout=10) for _ in range(2))
    assert got == {0: 15.0, 1: 15.0}


@pytest.mark.parametrize("shape,k", [((16, 24), 1), ((16, 24), 2), ((20, 8), 4)])
def test_block_columns_match_the_block_matrix_of_the_scan_geometry(shape, k):
    """The bench's on-device frame layout equals prep.frames_to_blockmatrix for the default
    geometry of rectangular frames and every knot spacing of the ragged workload."""
    import numpy as np
    import torch
    sys.path.insert(0, ROOT)
    import bench
    from steadyscan_b200 import prep
    h, w = shape
    img = np.arange(h * w, dtype=np.float64).reshape(h, w)
    s = prep.init_settings({"nknots": h // k + 1}, np.zeros((h + 4, w + 4)), h, w)
    lay = prep.block_layout(s)
    ref = prep.frames_to_blockmatrix(img, lay)
    got = bench.to_block_columns(torch.tensor(img), k).numpy().reshape(lay.frame_h, lay.frame_w, order="F")
    np.testing.assert_array_equal(got, ref)


def test_ragged_workload_shapes():
    """The ragged generator draws frame sizes, knot spacings and group lengths from their sets."""
    import torch  # noqa: F401
    sys.path.insert(0, ROOT)
    import bench
    groups, dev, meta = bench.make_ragged_workload("S", 7, "cpu", n_groups=3)
    assert len(groups) == len(dev) == len(meta) == 3
    for g, (t, lay), (h, w, k, nf) in zip(groups, dev, meta):
        assert (h, w) in [(128, 128), (256, 512), (512, 512), (796, 512)] and k in (1, 2, 4) and 1 <= nf <= 128
        assert g["bmData"].shape == (k * w, (h // k) * nf)
        assert t.numel() == h * w * nf
        assert g["move_thresh"] == 1e-3 and g["max_iter"] == 30
