"""Host logic of the serving loop on CPU: the device-memory pool that sizes admission, the arrival
schedule of the load generator and the latency statistics."""
import numpy as np

from steadyscan_b200 import serving


def test_pool_first_fit_alignment_and_merge():
    pool = serving.DevicePool(4096, "cpu")
    a = pool.alloc(100)
    b = pool.alloc(300)
    c = pool.alloc(256)
    assert a == (0, 256) and b == (256, 512) and c == (768, 256)
    assert all(off % serving.DevicePool.ALIGN == 0 for off, _ in (a, b, c))
    assert pool.used() == 1024
    pool.release(b)
    assert pool.alloc(200) == (256, 256)  # first fit reuses the hole
    assert pool.alloc(4096) is None       # larger than what is left: the request waits
    for blk in ((0, 256), (256, 256), (768, 256)):
        pool.release(blk)
    assert pool.free == [(0, 4096)] and pool.used() == 0  # neighbours merge back into one block


def test_arrival_schedule_rates_bursts_and_lengths():
    rng = np.random.default_rng(3)
    sched = serving.arrival_schedule(4, 100.0, 30.0, 10.0, 2.0, 2.0, (1, 64), rng)
    t = np.array([s[0] for s in sched])
    assert np.all(np.diff(t) >= 0) and t.min() >= 0 and t.max() < 100.0
    assert {s[1] for s in sched} == {0, 1, 2, 3}
    n = np.array([s[2] for s in sched])
    assert n.min() >= 1 and n.max() <= 64
    in_burst = (t % 10.0) < 2.0
    rate_burst = in_burst.sum() / (4 * 20.0)
    rate_calm = (~in_burst).sum() / (4 * 80.0)
    assert 45 < rate_burst < 75 and 24 < rate_calm < 36  # 60 and 30 per second per session


def test_latency_stats():
    class R:
        def __init__(self, lat, n):
            self.latency, self.n_frames = lat, n
    rs = [R(0.001 * (i + 1), 2) for i in range(100)]
    st = serving.latency_stats(rs)
    assert st["groups"] == 100 and st["frames"] == 200
    assert abs(st["p50_ms"] - 50.5) < 1e-9 and abs(st["p99_ms"] - 99.01) < 1e-9 and st["max_ms"] == 100.0
