"""Encode serving on one GPU: continuous batching of live encode sessions.

Sessions (a resolution, a quantizer, a length, a content seed) arrive over
time. Each is admitted as soon as a device-memory budget allows: its encoder
(libmav1.so, device state resident in HBM) joins the ones already running,
and its frames are coded concurrently with theirs — the device interleaves
every session's stage kernels, the process-wide host pool entropy-codes
whichever frames are ready. Frames of a session arrive in real time (30 per
second from its arrival); a frame's latency is the time from its arrival to
the moment its temporal unit comes out of the encoder. Sessions that cannot
be admitted wait in arrival order; the frames they receive meanwhile queue
up, so their latency includes the wait.

Encoders are kept when their session ends and reused by the next session of
the same frame size (mav1_cuda_restart: new quantizer and content, key frame
first, the bitstream of a fresh encoder). Creating and freeing device memory
synchronises the whole GPU, which would stall every running session; a pool
keeps the device state resident and only grows it. Idle pooled encoders
count against the budget and are freed first when a session of another size
needs room.

The reference has nothing like this (its API codes one stream per encoder);
the queue API it serves from is mav1.h's (mav1_send_frame / mav1_receive_
packet_wait, src/mav1.h:54-81; encoder.c:1295-1396).
"""
import dataclasses
import hashlib
import threading
import time

import numpy as np

import mav1api
import mav1cu
import synthetic

FPS = 30.0


@dataclasses.dataclass
class Session:
    sid: int
    arrival: float            # seconds after the start of the run
    width: int
    height: int
    q: int
    frames: int
    clip: np.ndarray = None   # [k, packed I420 bytes]: the content, played forward and back
    # results
    admitted: float = None
    done: float = None
    latencies: list = None    # per shown frame, seconds
    ivf_sha256: str = None
    error: str = None

    def frame(self, i):
        k = len(self.clip)
        period = max(1, 2 * k - 2)
        j = i % period
        return self.clip[j if j < k else period - j]

    def config(self):
        return mav1cu.cli_config(self.width, self.height, q=self.q, turbo=1)


def content_specs(per_size=2, frames=16, sizes=((640, 360), (1280, 720), (1920, 1080), (3840, 2160))):
    """Content clips per frame size: the 352x288 recipe scaled to the size
    (as synthetic.batch_streams), `per_size` seeds each."""
    specs = {}
    rng = np.random.default_rng(77)
    for (w, h) in sizes:
        s = w / 352.0
        specs[(w, h)] = [synthetic.ClipSpec(w, h, frames, seed=int(rng.integers(1, 1 << 30)), pan=(1.25 * s, -0.5 * s),
                                            rects=int(round(4 * s)),
                                            rect_size=(int(round(24 * s)), int(round(64 * s))),
                                            name=f"serve_{w}x{h}_{k}")
                         for k in range(per_size)]
    return specs


def poisson_sessions(n, rate, seed=1, mix=((640, 360, 0.3), (1280, 720, 0.4), (1920, 1080, 0.25), (3840, 2160, 0.05)),
                     length=(30, 300), qrange=(60, 200)):
    """n sessions with exponential inter-arrival times (rate per second),
    resolution drawn from the mix, length uniform in `length` frames, q
    uniform in `qrange`."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    sizes = [(w, h) for w, h, _ in mix]
    p = np.array([f for _, _, f in mix], float)
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        w, h = sizes[int(rng.choice(len(sizes), p=p / p.sum()))]
        out.append(Session(i, t, w, h, int(rng.integers(qrange[0], qrange[1] + 1)),
                           int(rng.integers(length[0], length[1] + 1))))
    return out


def mean_pixels_per_second(mix=((640, 360, 0.3), (1280, 720, 0.4), (1920, 1080, 0.25), (3840, 2160, 0.05)),
                           length=(30, 300)):
    """Expected pixels one session asks for per second of the run, per
    session-second (30 frames of its size)."""
    return FPS * sum(w * h * f for w, h, f in mix)


class Server:
    """Admits sessions against a device-memory budget and runs each admitted
    session's live encode on its own host thread."""

    def __init__(self, budget_bytes=150e9, max_active=256):
        self.budget = budget_bytes
        self.max_active = max_active
        self.cv = threading.Condition()
        self.pool = {}          # (w, h) -> [idle encoders]
        self.in_use = 0         # device bytes of active and pooled encoders
        self.active = 0
        self.peak_active = 0
        self.peak_bytes = 0
        self.encoders_created = 0

    # ---- encoder pool (under self.cv) ----
    def _take(self, s):
        idle = self.pool.get((s.width, s.height))
        if idle:
            return idle.pop()
        need = mav1api.device_bytes_for(s.config())
        while self.in_use + need > self.budget:
            # free an idle encoder of another size
            victim = next(((k, v) for k, v in self.pool.items() if v), None)
            if victim is None:
                return None
            e = victim[1].pop()
            self.in_use -= e.device_bytes()
            e.close()
        e = mav1api.Encoder(s.config())
        self.encoders_created += 1
        self.in_use += e.device_bytes()
        self.peak_bytes = max(self.peak_bytes, self.in_use)
        return e

    def _give_back(self, s, e):
        self.pool.setdefault((s.width, s.height), []).append(e)

    def _admissible(self, s):
        if self.active >= self.max_active:
            return False
        if self.pool.get((s.width, s.height)):
            return True
        need = mav1api.device_bytes_for(s.config())
        idle = sum(e.device_bytes() for v in self.pool.values() for e in v)
        return self.in_use - idle + need <= self.budget

    # ---- one session ----
    def _run_session(self, s, enc, t0):
        try:
            enc.restart(s.config())
            recv = []
            packets = []

            def drain(wait_ms=None):
                while True:
                    r = enc.receive(recon=False, wait_ms=wait_ms)
                    if r is None:
                        return
                    recv.append(time.perf_counter() - t0)
                    packets.append(r[0])

            for i in range(s.frames):
                due = s.arrival + i / FPS
                lag = due - (time.perf_counter() - t0)
                if lag > 0:
                    time.sleep(lag)
                enc.send(s.frame(i))
                drain()
            enc.send(None)
            while len(packets) < s.frames:
                n = len(packets)
                drain(wait_ms=100)
                if len(packets) == n and not enc.busy():
                    break
            if len(packets) != s.frames:
                raise RuntimeError(f"session {s.sid}: {len(packets)} of {s.frames} temporal units")
            s.latencies = [recv[k] - (s.arrival + k / FPS) for k in range(s.frames)]
            s.ivf_sha256 = hashlib.sha256(mav1api.ivf_bytes(packets, s.width, s.height)).hexdigest()
        except Exception as ex:  # reported in the results
            s.error = repr(ex)
        finally:
            s.done = time.perf_counter() - t0
            with self.cv:
                self._give_back(s, enc)
                self.active -= 1
                self.cv.notify_all()

    def run(self, sessions):
        """Serves the sessions (sorted by arrival) in real time; returns the
        run's wall-clock seconds."""
        sessions = sorted(sessions, key=lambda x: x.arrival)
        t0 = time.perf_counter()
        waiting, threads, nxt = [], [], 0
        with self.cv:
            while nxt < len(sessions) or waiting or self.active:
                now = time.perf_counter() - t0
                while nxt < len(sessions) and sessions[nxt].arrival <= now:
                    waiting.append(sessions[nxt])
                    nxt += 1
                while waiting and self._admissible(waiting[0]):
                    s = waiting.pop(0)
                    enc = self._take(s)
                    if enc is None:
                        waiting.insert(0, s)
                        break
                    s.admitted = time.perf_counter() - t0
                    self.active += 1
                    self.peak_active = max(self.peak_active, self.active)
                    th = threading.Thread(target=self._run_session, args=(s, enc, t0), daemon=True)
                    th.start()
                    threads.append(th)
                if nxt < len(sessions):
                    timeout = max(0.0, sessions[nxt].arrival - (time.perf_counter() - t0))
                    self.cv.wait(timeout=min(timeout, 0.05))
                elif waiting or self.active:
                    self.cv.wait(timeout=0.05)
        for th in threads:
            th.join()
        return time.perf_counter() - t0

    def close(self):
        with self.cv:
            for v in self.pool.values():
                for e in v:
                    e.close()
            self.pool = {}
            self.in_use = 0


def summary(sessions, wall):
    lat = np.concatenate([np.asarray(s.latencies) for s in sessions if s.latencies])
    frames = sum(s.frames for s in sessions if s.latencies)
    return {"sessions": len(sessions), "failed": sum(1 for s in sessions if s.error),
            "frames": int(frames), "wall_s": round(wall, 2), "fps": round(frames / wall, 1),
            "latency_ms_p50": round(1e3 * float(np.percentile(lat, 50)), 2),
            "latency_ms_p99": round(1e3 * float(np.percentile(lat, 99)), 2),
            "latency_ms_max": round(1e3 * float(lat.max()), 2),
            "admission_wait_ms_p99": round(1e3 * float(np.percentile(
                [s.admitted - s.arrival for s in sessions if s.admitted is not None], 99)), 2)}
