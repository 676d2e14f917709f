"""The batching and serving layers on the GPU: many streams of uneven size
coded at once, and live sessions admitted against a memory budget, must
give every stream the bitstream it gets alone (and the oracle's, for the
streams checked against it)."""
import hashlib

import numpy as np
import pytest

import batch
import mav1api
import mav1cu
import oracle
import serve
import synthetic

pytestmark = pytest.mark.gpu


def _h(b):
    return hashlib.sha256(b).hexdigest()


def _ivf(packets, w, h):
    return _h(mav1api.ivf_bytes(packets, w, h))


def test_batch_concurrent_equals_alone_and_oracle():
    """Four streams of three sizes and quantizers coded at once, twice on the
    same live encoders (each pass a new closed GOP), against each stream
    coded alone by a fresh encoder and, for two of them, by the oracle."""
    specs = [(synthetic.ClipSpec(352, 288, 10, seed=61, rects=3), 80),
             (synthetic.ClipSpec(640, 360, 10, seed=62, pan=(2.3, -0.9), rects=6, rect_size=(40, 110)), 170),
             (synthetic.ClipSpec(352, 288, 10, seed=63, rects=2), 125),
             (synthetic.ClipSpec(1280, 720, 10, seed=64, pan=(4.5, -1.8), rects=12, rect_size=(80, 220)), 125)]
    frames = [synthetic.packed_clip(s) for s, _ in specs]
    cfgs = [mav1cu.cli_config(s.width, s.height, q=q, turbo=1, keyint=s.frames) for s, q in specs]
    B = batch.Batch(list(zip(cfgs, frames)))
    try:
        _, first = B.code(concurrent=True)
        _, second = B.code(concurrent=True)
        _, seq = B.code(concurrent=False)
    finally:
        B.close()
    for (s, q), a, b, c, f, cfg in zip(specs, first, second, seq, frames, cfgs):
        alone, _ = mav1api.encode(list(f), cfg, recon=False)
        want = _ivf(alone, s.width, s.height)
        assert _ivf(a[0], s.width, s.height) == want
        assert _ivf(b[0], s.width, s.height) == want
        assert _ivf(c[0], s.width, s.height) == want
    if oracle.available():
        for (s, q), a in list(zip(specs, first))[:2]:
            pk, _ = oracle.encode(list(synthetic.generate(s)), oracle.cli_config(s.width, s.height, q=q, turbo=1))
            assert oracle.ivf_bytes(pk, s.width, s.height) == mav1api.ivf_bytes(a[0], s.width, s.height)


def _sessions():
    specs = {(352, 288): [synthetic.ClipSpec(352, 288, 8, seed=71, rects=3)],
             (640, 360): [synthetic.ClipSpec(640, 360, 8, seed=72, pan=(2.3, -0.9), rects=6, rect_size=(40, 110))]}
    clips = {k: synthetic.packed_clip(v[0]) for k, v in specs.items()}
    rng = np.random.default_rng(5)
    out = []
    for i in range(6):
        w, h = (352, 288) if i % 3 else (640, 360)
        s = serve.Session(i, 0.05 * i, w, h, int(rng.integers(60, 201)), int(rng.integers(14, 30)))
        s.clip = clips[(w, h)]
        out.append(s)
    return out


def test_serving_alone_equals_mix():
    """Six live sessions of two sizes arriving 50 ms apart, served together:
    each session's bitstream equals the one it gets alone, encoders are
    reused across sessions of one size, and the frame latencies are
    recorded."""
    sessions = _sessions()
    srv = serve.Server(budget_bytes=150e9)
    try:
        srv.run(sessions)
    finally:
        srv.close()
    assert all(s.error is None for s in sessions), [s.error for s in sessions]
    assert srv.peak_active >= 2
    for s in sessions:
        assert len(s.latencies) == s.frames and min(s.latencies) > 0
        pk, _ = mav1api.encode([s.frame(i) for i in range(s.frames)], s.config(), recon=False)
        assert _ivf(pk, s.width, s.height) == s.ivf_sha256, s.sid
    if oracle.available():
        s = sessions[1]
        frames = []
        for i in range(s.frames):
            f = np.asarray(s.frame(i))
            y, u, v = np.split(f, [s.width * s.height, s.width * s.height + (s.width // 2) * (s.height // 2)])
            frames.append([y.reshape(s.height, s.width), u.reshape(s.height // 2, -1), v.reshape(s.height // 2, -1)])
        pk, _ = oracle.encode(frames, oracle.cli_config(s.width, s.height, q=s.q, turbo=1))
        assert _h(oracle.ivf_bytes(pk, s.width, s.height)) == s.ivf_sha256


def test_serving_admission_respects_budget():
    """With a budget that fits one encoder, sessions are served one at a
    time (the others wait in arrival order) and every one completes."""
    sessions = _sessions()[:3]
    for s in sessions:
        s.width, s.height = 352, 288
        s.clip = synthetic.packed_clip(synthetic.ClipSpec(352, 288, 8, seed=71, rects=3))
    one = mav1api.device_bytes_for(sessions[0].config())
    srv = serve.Server(budget_bytes=one * 1.5)
    try:
        srv.run(sessions)
    finally:
        srv.close()
    assert all(s.error is None for s in sessions)
    assert srv.peak_active == 1 and srv.encoders_created == 1
    assert sessions[2].admitted >= sessions[1].done - 1e-3


def test_device_bytes_prediction_matches_allocation():
    for w, h in [(352, 288), (203, 131), (1920, 1080)]:
        cfg = mav1cu.cli_config(w, h, q=100, turbo=1)
        e = mav1api.Encoder(cfg)
        try:
            assert e.device_bytes() == mav1api.device_bytes_for(cfg)
        finally:
            e.close()
