"""Serving loop: frame groups from several imaging sessions aligned together on one GPU.

The reference aligns one group per synchronous MEX call (steady_scan.m:216-287). Here groups are
served by continuous batching (``ss_server_*``):

* a session (``api.Session``) holds its template, gradients and scan geometry on the device, and
  the server remembers its last displacements, the warm start of its next group;
* a request is one group of frames; it is admitted into a free slot of the engine's server when a
  device memory pool (the budget) has room for its buffers (``api.Batch.measure``);
* the engine runs every active group's next cycle with one launch sequence; between cycles groups
  that stopped leave (their outputs collected, memory returned) and admitted ones join, so requests
  arriving while others run are served together with them.

Each request's result is the one its group gets alone: the kernels only read shared session
buffers and every group's state machine is its own.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field

import numpy as np

from . import api
from ._lib import check, load


class DevicePool:
    """First-fit allocator of 256-byte aligned blocks in one device buffer (the memory budget)."""

    ALIGN = 256

    def __init__(self, nbytes: int, device):
        import torch
        self.buf = torch.empty(int(nbytes), dtype=torch.uint8, device=device)
        self.base = self.buf.data_ptr()
        self.size = int(nbytes)
        self.free = [(0, self.size)]  # sorted (offset, length)

    def alloc(self, n: int):
        n = (int(n) + self.ALIGN - 1) // self.ALIGN * self.ALIGN
        for k, (off, ln) in enumerate(self.free):
            a = (off + self.ALIGN - 1) // self.ALIGN * self.ALIGN
            if a + n <= off + ln:
                rest = []
                if a > off:
                    rest.append((off, a - off))
                if a + n < off + ln:
                    rest.append((a + n, off + ln - a - n))
                self.free[k:k + 1] = rest
                return a, n
        return None

    def release(self, block):
        off, n = block
        self.free.append((off, n))
        self.free.sort()
        merged = []
        for o, ln in self.free:
            if merged and merged[-1][0] + merged[-1][1] == o:
                merged[-1] = (merged[-1][0], merged[-1][1] + ln)
            else:
                merged.append((o, ln))
        self.free = merged

    def used(self) -> int:
        return self.size - sum(ln for _, ln in self.free)


@dataclass
class SessionState:
    sid: int
    proto: dict
    session: api.Session
    last_knots: tuple | None = None  # (dx, dy) of the latest group that aligned well, its last frame
    memo: dict = field(default_factory=dict)  # converted template / geometry matrices, reused per request
    keep: list = field(default_factory=list)


@dataclass
class Request:
    rid: int
    sid: int
    frames: object               # block-matrix frames: host array or api.DeviceMatrix
    n_frames: int
    t_arrival: float
    est_dx: np.ndarray | None = None
    est_dy: np.ndarray | None = None
    args: dict | None = None
    block: tuple | None = None
    slot: int = -1
    need: int = 0                # device bytes of the group's buffers
    t_admit: float = 0.0
    t_done: float = 0.0
    result: dict | None = None
    in_burst: bool = False       # caller's label for latency reports (e.g. arrived during a load burst)
    _c: tuple | None = None      # ctypes inputs/outputs kept alive while the group runs

    @property
    def latency(self) -> float:
        return self.t_done - self.t_arrival


@dataclass
class Server:
    """Continuous-batching server over ``memory_budget`` bytes of device memory and at most
    ``max_active`` groups in flight."""
    memory_budget: int
    device: int = 0
    max_active: int = 64
    warm_start: bool = True
    sessions: list = field(default_factory=list)
    pending: list = field(default_factory=list)
    done: list = field(default_factory=list)

    def __post_init__(self):
        import torch
        self._lib = load()
        self.pool = DevicePool(self.memory_budget, torch.device("cuda", self.device))
        h = C.c_void_p()
        check(self._lib.ss_server_create(self.max_active, self.device, C.byref(h)))
        self._h = h
        self.by_slot: dict = {}
        self._next = 0
        self.peak_active = 0
        self.peak_bytes = 0
        self.cycles = 0
        self._done_buf = (C.c_int32 * self.max_active)()

    @property
    def active(self) -> list:
        return list(self.by_slot.values())

    def add_session(self, proto: dict, template_storage=None) -> int:
        """Registers a session from an argument dict (template, gradients, geometry, settings)."""
        sid = len(self.sessions)
        p = dict(proto)
        p["gpu_device_id"] = self.device
        st = SessionState(sid, p, api.Session(p, template_storage))
        # the requests pass these same arrays: convert them once (the library reads only their shapes)
        _, st.keep = api._inputs(p, template_storage, st.memo)
        self.sessions.append(st)
        return sid

    def submit(self, sid: int, frames, n_frames: int, t_arrival: float | None = None, est_dx=None,
               est_dy=None) -> Request:
        """Queues a group of ``n_frames`` frames of session ``sid``; initial knots default to the
        session's warm start."""
        r = Request(self._next, sid, frames, int(n_frames), time.perf_counter() if t_arrival is None else t_arrival,
                    est_dx, est_dy)
        self._next += 1
        self.pending.append(r)
        return r

    # --------------------------------------------------------------------------------------------

    def _group_args(self, r: Request, admit: bool) -> dict:
        """The group's argument dict; on admission the initial knots are fixed (the caller's, else
        the session's warm start as it stands then, else zeros)."""
        st = self.sessions[r.sid]
        a = dict(st.proto)
        w1 = a["tfrac"].shape[1] + 1
        ex, ey = r.est_dx, r.est_dy
        if ex is None:
            if self.warm_start and st.last_knots is not None:
                # the displacement where the session's last group ended, for every knot: the guess
                # of a drifting displacement a moment later
                ex = np.full((w1, r.n_frames), st.last_knots[0])
                ey = np.full((w1, r.n_frames), st.last_knots[1])
            else:
                ex = np.zeros((w1, r.n_frames))
                ey = np.zeros((w1, r.n_frames))
            if admit:
                r.est_dx, r.est_dy = ex, ey
        a["bmData"] = r.frames
        a["nFrames"] = r.n_frames
        a["est_dx_knots"] = np.asfortranarray(ex)
        a["est_dy_knots"] = np.asfortranarray(ey)
        return a

    def _admit(self):
        while self.pending and len(self.by_slot) < self.max_active:
            r = self.pending[0]
            st = self.sessions[r.sid]
            ses = st.session
            ts = ses.template_storage
            if not r.need:
                r.need = api.Batch.measure([self._group_args(r, False)], template_storage=ts, sessions=[ses],
                                           memo=st.memo)
            block = self.pool.alloc(r.need)
            if block is None:
                break  # waits for memory to free up
            self.pending.pop(0)
            a = self._group_args(r, True)
            i, keep = api._inputs(a, ts, st.memo)
            o, arrays, dims = api._outputs(a, False, False)
            slot = C.c_int32(-1)
            rc = self._lib.ss_server_admit(self._h, C.byref(i), C.byref(o), ses.handle, self.pool.base + block[0],
                                           block[1], C.byref(slot))
            if rc:
                self.pool.release(block)
                check(rc)
            r.args, r.block, r.slot, r.t_admit = a, block, slot.value, time.perf_counter()
            r._c = (i, keep, o, arrays, dims)
            self.by_slot[r.slot] = r
        self.peak_active = max(self.peak_active, len(self.by_slot))
        self.peak_bytes = max(self.peak_bytes, self.pool.used())

    def _retire(self, slot: int):
        r = self.by_slot.pop(slot)
        i, keep, o, arrays, dims = r._c
        r.result = api._result(o, arrays, dims)
        r.t_done = time.perf_counter()
        r._c = None
        self.pool.release(r.block)
        st = self.sessions[r.sid]
        # warm start: the median of the last frame's knots without its last two (the chain's last
        # knot is never solved, and the last block column is bounded by a fixed knot); a group that
        # did not align (low correlation) leaves the warm start as it was
        w1 = r.args["tfrac"].shape[1] + 1
        dx = np.asarray(r.result["dx"])[-w1:-2]
        dy = np.asarray(r.result["dy"])[-w1:-2]
        corr = np.asarray(r.result["frame_corr"], dtype=np.float64)
        if dx.size and np.all(np.isfinite(corr)) and float(np.mean(corr)) >= 0.5:
            st.last_knots = (float(np.median(dx)), float(np.median(dy)))
        self.done.append(r)

    def tick(self) -> int:
        """One pass of the loop: once the cycle in flight has finished, retire the groups that
        stopped and launch the next cycle; then admit queued requests while the GPU works (they join
        at the following cycle). Returns the number of groups in the server."""
        n = C.c_int32(0)
        rc = self._lib.ss_server_poll(self._h, self._done_buf, self.max_active, C.byref(n))
        if rc < 0:
            check(rc)
        if rc == 1:
            for k in range(n.value):
                self._retire(self._done_buf[k])
            if self.by_slot:
                check(self._lib.ss_server_step(self._h))
                self.cycles += 1
        self._admit()
        return len(self.by_slot)

    def drain(self, timeout_s: float = 600.0):
        t_end = time.perf_counter() + timeout_s
        while (self.by_slot or self.pending) and time.perf_counter() < t_end:
            self.tick()
        if self.by_slot or self.pending:
            raise TimeoutError("serving queue did not drain")

    def close(self):
        if getattr(self, "_h", None):
            self._lib.ss_server_destroy(self._h)
            self._h = None
        for s in self.sessions:
            s.session.close()


def latency_stats(requests) -> dict:
    lat = np.array([r.latency for r in requests]) * 1000.0
    fr = sum(r.n_frames for r in requests)
    return {"groups": len(requests), "frames": int(fr),
            "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
            "max_ms": float(lat.max()) if len(lat) else None}


def arrival_schedule(n_sessions: int, duration_s: float, rate_hz: float, burst_every_s: float, burst_len_s: float,
                     burst_factor: float, group_len: tuple, rng) -> list:
    """Poisson arrivals per session at rate_hz, multiplied by burst_factor for burst_len_s at the
    start of every burst_every_s; group lengths uniform in group_len. Returns sorted
    (t, session, n_frames)."""
    out = []
    for s in range(n_sessions):
        t = 0.0
        while True:
            in_burst = (t % burst_every_s) < burst_len_s
            t += rng.exponential(1.0 / (rate_hz * (burst_factor if in_burst else 1.0)))
            if t >= duration_s:
                break
            out.append((t, s, int(rng.integers(group_len[0], group_len[1] + 1))))
    out.sort()
    return out
