"""Serving loop: requests of several sessions in flight together give their alone results."""
import numpy as np
import pytest

from steadyscan_b200 import api, serving
from tests.helpers import make_args

pytestmark = pytest.mark.gpu


def _sessions():
    recs = []
    for seed, kw in ((81, dict(nlines=32, linewidth=32, nknots=9)), (82, dict(nlines=64, linewidth=64, nknots=33))):
        args, _, _ = make_args(n_frames=12, seed=seed, frame_dtype=np.uint16, n_blobs=20, **kw)
        args["flags"] = "S"
        recs.append(args)
    return recs


def _requests(recs, server, sizes):
    out = []
    for k, n in enumerate(sizes):
        sid = k % len(recs)
        a = recs[sid]
        w = a["tfrac"].shape[1]
        f0 = (3 * k) % (12 - n + 1)
        frames = np.asfortranarray(np.asarray(a["bmData"])[:, f0 * w:(f0 + n) * w])
        out.append(server.submit(sid, frames, n))
    return out


def test_requests_in_the_mix_equal_their_alone_results():
    """Groups of two sessions (different template and frame sizes) run in one server, joining and
    leaving between cycles; each group's knots and iteration count equal those of aligning the same
    group (same frames, same initial knots) alone."""
    recs = _sessions()
    server = serving.Server(memory_budget=512 << 20)
    try:
        for a in recs:
            server.add_session(a)
        reqs = _requests(recs, server, [3, 1, 4, 2, 4, 1, 2, 3])
        server.drain()
        assert server.peak_active >= 2  # several requests were in flight together
        for r in reqs:
            alone = api.align_group(r.args, want_mask=False)
            assert alone["iter_used"] == r.result["iter_used"]
            np.testing.assert_array_equal(alone["dx"], r.result["dx"])
            np.testing.assert_array_equal(alone["dy"], r.result["dy"])
    finally:
        server.close()


def test_memory_budget_admits_one_request_at_a_time():
    """A memory budget of one group's buffers admits one request at a time, and each later request
    of the session starts from the displacement where the one before ended (warm start: the median
    of its last frame's knots but the last two)."""
    recs = _sessions()[:1]
    a = dict(recs[0])
    w = a["tfrac"].shape[1]
    a["bmData"] = np.asfortranarray(np.asarray(a["bmData"])[:, :4 * w])
    a["nFrames"] = 4
    a["est_dx_knots"] = np.zeros((w + 1, 4))
    a["est_dy_knots"] = np.zeros((w + 1, 4))
    server = serving.Server(memory_budget=1 << 30)
    try:
        sid = server.add_session(recs[0])
        need = api.Batch.measure([a], sessions=[server.sessions[sid].session])
        server.close()
        server = serving.Server(memory_budget=need + need // 2)
        server.add_session(recs[0])
        reqs = _requests(recs, server, [4, 4, 4])
        server.drain()
        assert server.peak_active == 1
        assert len(server.done) == 3
        for prev, cur in zip(reqs, reqs[1:]):
            assert np.all(cur.est_dx == np.median(np.asarray(prev.result["dx"])[-(w + 1):-2]))
            assert np.all(cur.est_dy == np.median(np.asarray(prev.result["dy"])[-(w + 1):-2]))
    finally:
        server.close()
