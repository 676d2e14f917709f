"""The batching and serving layers' host logic on CPU: a fake encoder with
the mav1api.Encoder interface stands in for libmav1.so (no device), so the
admission against the memory budget, the encoder pool (reuse by frame size,
eviction of idle encoders of other sizes), arrival order, per-frame latency
accounting, error reporting and the batch's stream bookkeeping are checked
without a GPU. Its packets are a digest of the session's configuration, the
frame index and the frame's bytes, so a frame routed to the wrong encoder,
out of order or twice changes a stream's hash."""
import hashlib
import threading

import numpy as np
import pytest

import batch
import mav1api
import mav1cu
import serve

BYTES_PER_PIXEL = 100  # the fake's device bytes per luma sample


class FakeEncoder:
    live_bytes = 0
    peak_bytes = 0
    created = []
    lock = threading.Lock()
    fail_q = None  # sessions with this quantizer raise on their third frame

    def __init__(self, cfg):
        c = np.ascontiguousarray(cfg)[0]
        self.w, self.h = int(c["width"]), int(c["height"])
        self.size = self.w * self.h + 2 * ((self.w + 1) // 2) * ((self.h + 1) // 2)
        self.cfg = np.ascontiguousarray(cfg).copy()
        self.n = 0
        self.out = []
        self.closed = False
        with FakeEncoder.lock:
            FakeEncoder.live_bytes += self.device_bytes()
            FakeEncoder.peak_bytes = max(FakeEncoder.peak_bytes, FakeEncoder.live_bytes)
            FakeEncoder.created.append(self)

    @classmethod
    def reset(cls):
        cls.live_bytes = cls.peak_bytes = 0
        cls.created = []
        cls.fail_q = None

    def device_bytes(self):
        return self.w * self.h * BYTES_PER_PIXEL

    def restart(self, cfg):
        c = np.ascontiguousarray(cfg)[0]
        assert (int(c["width"]), int(c["height"])) == (self.w, self.h), "restart with another frame size"
        self.cfg = np.ascontiguousarray(cfg).copy()
        self.n = 0
        self.out = []

    def send(self, frame):
        assert not self.closed
        if frame is None:
            return
        a = np.ascontiguousarray(frame, np.uint8).reshape(-1)
        if a.size != self.size:
            raise mav1api.Mav1Error(f"frame of {a.size} bytes, expected {self.size}")
        if FakeEncoder.fail_q is not None and int(self.cfg[0]["qindex"]) == FakeEncoder.fail_q and self.n == 2:
            raise mav1api.Mav1Error("injected failure")
        # closed GOPs: with a key-frame interval, every interval codes alike
        keyint = int(self.cfg[0]["keyint"])
        idx = self.n % keyint if keyint > 0 else self.n
        self.out.append(hashlib.sha256(self.cfg.tobytes() + idx.to_bytes(4, "little") + a.tobytes()).digest())
        self.n += 1

    def receive(self, recon=True, wait_ms=None):
        if not self.out:
            return None
        return self.out.pop(0), None

    def busy(self):
        return 0

    def close(self):
        if not self.closed:
            self.closed = True
            with FakeEncoder.lock:
                FakeEncoder.live_bytes -= self.device_bytes()


@pytest.fixture
def fake(monkeypatch):
    FakeEncoder.reset()
    monkeypatch.setattr(mav1api, "Encoder", FakeEncoder)
    monkeypatch.setattr(mav1api, "device_bytes_for",
                        lambda cfg: int(cfg[0]["width"]) * int(cfg[0]["height"]) * BYTES_PER_PIXEL)
    yield FakeEncoder
    FakeEncoder.reset()


def _clip(w, h, k, seed):
    rng = np.random.default_rng(seed)
    n = w * h + 2 * ((w + 1) // 2) * ((h + 1) // 2)
    return rng.integers(0, 256, (k, n), dtype=np.uint8)


def _session(sid, t, w, h, q, frames, seed):
    s = serve.Session(sid, t, w, h, q, frames)
    s.clip = _clip(w, h, 3, seed)
    return s


def _serve(sessions, budget):
    srv = serve.Server(budget_bytes=budget)
    try:
        wall = srv.run(sessions)
    finally:
        stats = (srv.peak_active, srv.peak_bytes, srv.encoders_created)
        srv.close()
    return wall, stats


def test_admission_keeps_to_the_budget_and_reuses_encoders(fake):
    one = 64 * 48 * BYTES_PER_PIXEL
    sessions = [_session(i, 0.02 * i, 64, 48, 100 + i, 4, seed=i) for i in range(5)]
    _, (peak_active, peak_bytes, created) = _serve(sessions, budget=2 * one)
    assert all(s.error is None for s in sessions), [s.error for s in sessions]
    assert peak_active == 2 and created == 2 and len(fake.created) == 2
    assert peak_bytes <= 2 * one and fake.peak_bytes <= 2 * one
    # the third session starts only once one of the first two has ended
    assert sessions[2].admitted >= min(sessions[0].done, sessions[1].done) - 1e-3
    for s in sessions:
        assert len(s.latencies) == s.frames
        assert s.admitted >= s.arrival - 1e-3
        # a frame comes out after it arrives, and a waiting session's first frame waits for admission
        assert min(s.latencies) >= -1e-3 and s.latencies[0] >= s.admitted - s.arrival - 5e-3
    # every session's stream is the one it gets alone on the server
    for s in sessions:
        alone = _session(s.sid, 0.0, s.width, s.height, s.q, s.frames, seed=s.sid)
        _serve([alone], budget=one)
        assert alone.ivf_sha256 == s.ivf_sha256


def test_idle_encoders_of_another_size_are_freed_for_a_new_session(fake):
    small, large = 64 * 48 * BYTES_PER_PIXEL, 128 * 96 * BYTES_PER_PIXEL
    sessions = [_session(0, 0.0, 64, 48, 90, 3, seed=1), _session(1, 0.0, 64, 48, 91, 3, seed=2),
                _session(2, 0.3, 128, 96, 92, 3, seed=3)]
    _, (peak_active, peak_bytes, created) = _serve(sessions, budget=large)
    assert all(s.error is None for s in sessions)
    assert created == 3 and peak_bytes <= large and 2 * small <= large
    small_encs = [e for e in fake.created if e.w == 64]
    assert len(small_encs) == 2 and all(e.closed for e in small_encs)  # evicted, not kept beside the large one
    assert sessions[2].admitted >= 0.3 - 1e-3


def test_waiting_sessions_are_admitted_in_arrival_order(fake):
    small, large = 64 * 48 * BYTES_PER_PIXEL, 128 * 96 * BYTES_PER_PIXEL
    sessions = [_session(0, 0.0, 128, 96, 80, 4, seed=4), _session(1, 0.01, 128, 96, 81, 4, seed=5),
                _session(2, 0.02, 64, 48, 82, 2, seed=6)]
    _serve(sessions, budget=large + small)
    assert all(s.error is None for s in sessions)
    # the second large session waits for the first; the small one would fit
    # beside the first but must not overtake the large one waiting before it
    assert sessions[1].admitted >= sessions[0].done - 1e-3
    assert sessions[2].admitted >= sessions[1].admitted and sessions[2].admitted >= sessions[0].done - 1e-3


def test_a_failing_session_is_reported_and_the_others_complete(fake):
    fake.fail_q = 77
    sessions = [_session(0, 0.0, 64, 48, 70, 4, seed=7), _session(1, 0.0, 64, 48, 77, 4, seed=8),
                _session(2, 0.01, 64, 48, 71, 4, seed=9)]
    wall, _ = _serve(sessions, budget=10 * 64 * 48 * BYTES_PER_PIXEL)
    assert sessions[1].error and "injected failure" in sessions[1].error and sessions[1].latencies is None
    assert sessions[0].error is None and sessions[2].error is None
    sm = serve.summary(sessions, wall)
    assert sm["sessions"] == 3 and sm["failed"] == 1 and sm["frames"] == 8
    lat = np.concatenate([sessions[0].latencies, sessions[2].latencies])
    assert sm["latency_ms_p50"] == round(1e3 * float(np.percentile(lat, 50)), 2)
    assert sm["latency_ms_p99"] == round(1e3 * float(np.percentile(lat, 99)), 2)


def test_poisson_arrivals():
    a = serve.poisson_sessions(4000, rate=5.0, seed=3)
    b = serve.poisson_sessions(4000, rate=5.0, seed=3)
    assert [(s.arrival, s.width, s.q, s.frames) for s in a] == [(s.arrival, s.width, s.q, s.frames) for s in b]
    gaps = np.diff([0.0] + [s.arrival for s in a])
    assert (gaps > 0).all() and abs(gaps.mean() - 0.2) < 0.02
    share = np.mean([s.width == 1280 for s in a])
    assert abs(share - 0.4) < 0.03
    assert all(30 <= s.frames <= 300 and 60 <= s.q <= 200 for s in a)


def test_batch_concurrent_equals_one_after_another(fake):
    sizes = [(64, 48), (96, 64), (64, 48)]
    streams = [(mav1cu.cli_config(w, h, q=100 + i, turbo=1, keyint=5), list(_clip(w, h, 5, seed=20 + i)))
               for i, (w, h) in enumerate(sizes)]
    B = batch.Batch(streams)
    try:
        _, conc = B.code(concurrent=True)
        _, again = B.code(concurrent=True)
        _, seq = B.code(concurrent=False)
    finally:
        B.close()
    assert len(fake.created) == 3 and all(e.closed for e in fake.created)
    hashes = []
    for (cfg, fr), a, b, c, (w, h) in zip(streams, conc, again, seq, sizes):
        assert len(a[0]) == len(fr)
        hashes.append(batch.stream_hashes(a, w, h))
        assert hashes[-1] == batch.stream_hashes(b, w, h) == batch.stream_hashes(c, w, h)
        # each stream's result is its own: coding it alone on a fresh encoder gives the same units
        alone = mav1api.code_frames(FakeEncoder(cfg), fr, len(fr), recon=False)
        assert alone[0] == a[0]
    assert len(set(hashes)) == 3


def test_batch_reraises_a_stream_failure(fake):
    fake.fail_q = 55
    streams = [(mav1cu.cli_config(64, 48, q=55, turbo=1), list(_clip(64, 48, 4, seed=30))),
               (mav1cu.cli_config(64, 48, q=56, turbo=1), list(_clip(64, 48, 4, seed=31)))]
    B = batch.Batch(streams)
    try:
        with pytest.raises(mav1api.Mav1Error, match="injected failure"):
            B.code(concurrent=True)
    finally:
        B.close()
