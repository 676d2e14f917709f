"""Seeded synthetic 8-bit 4:2:0 clips (the content of the encode benchmarks).

Recipe per plane (luma at full resolution, each chroma plane at half
resolution):
  1. a texture of uniform [0, 255] noise, Gaussian-blurred (periodic
     boundary) with sigma ``blur`` (luma) or ``blur_uv`` (chroma);
  2. a global pan of ``pan = (dx, dy)`` px per frame (halved for chroma),
     sampled from the periodic texture with bilinear sub-pixel resampling;
  3. ``rects`` opaque rectangles of flat value, side lengths uniform in
     ``rect_size``, values uniform in [30, 220], moving linearly with integer
     velocities in [-4, 4] px per frame; chroma uses the same rectangles with
     positions and sizes halved (floor) and its own flat values;
  4. per-frame Gaussian noise of sigma ``noise``, rounding and clipping to
     [0, 255].
An optional scene cut re-seeds everything from frame ``cut``.

Everything is float64 numpy from one ``numpy.random.default_rng(seed)``
stream, so a (config, seed) pair always yields the same bytes.
"""
from dataclasses import dataclass, field
import hashlib

import numpy as np


@dataclass
class ClipSpec:
    width: int
    height: int
    frames: int
    seed: int = 1
    blur: float = 3.0
    blur_uv: float = 5.0
    pan: tuple = (1.25, -0.5)
    rects: int = 4
    rect_size: tuple = (24, 64)
    noise: float = 2.0
    cut: int = -1            # frame index of a scene cut (-1: none)
    name: str = field(default="")


# The benchmark clips (seeded stand-ins for the reference's test content).
CONFIGS = {
    "c0_352x288": ClipSpec(352, 288, 30, seed=1, name="c0_352x288"),
    "c1_1080p": ClipSpec(1920, 1080, 120, seed=1, pan=(2.5, 1.0), rects=12, rect_size=(64, 256),
                         name="c1_1080p"),
    "c2_2160p": ClipSpec(3840, 2160, 32, seed=1, blur=4.0, rects=24, rect_size=(128, 512), cut=16,
                         name="c2_2160p"),
}


def _gauss_kernel(sigma):
    r = int(np.ceil(3 * sigma))
    x = np.arange(-r, r + 1, dtype=np.float64)
    k = np.exp(-0.5 * (x / sigma) ** 2)
    return k / k.sum()


def _blur_periodic(img, sigma):
    k = _gauss_kernel(sigma)
    r = len(k) // 2
    out = np.zeros_like(img)
    for i, w in enumerate(k):
        out += w * np.roll(img, i - r, axis=1)
    img = out
    out = np.zeros_like(img)
    for i, w in enumerate(k):
        out += w * np.roll(img, i - r, axis=0)
    return out


def _pan_sample(tex, h, w, ox, oy):
    th, tw = tex.shape
    ys = np.arange(h, dtype=np.float64) + oy
    xs = np.arange(w, dtype=np.float64) + ox
    y0 = np.floor(ys)
    x0 = np.floor(xs)
    fy = (ys - y0)[:, None]
    fx = (xs - x0)[None, :]
    y0 = y0.astype(np.int64) % th
    x0 = x0.astype(np.int64) % tw
    y1 = (y0 + 1) % th
    x1 = (x0 + 1) % tw
    r0 = tex.take(y0, axis=0)
    r1 = tex.take(y1, axis=0)
    a = r0.take(x0, axis=1)
    b = r0.take(x1, axis=1)
    c = r1.take(x0, axis=1)
    d = r1.take(x1, axis=1)
    return (a * (1 - fx) + b * fx) * (1 - fy) + (c * (1 - fx) + d * fx) * fy


class _Scene:
    def __init__(self, spec, rng):
        self.spec = spec
        w, h = spec.width, spec.height
        cw, ch = (w + 1) // 2, (h + 1) // 2
        tpad = 64
        self.tex = [
            _blur_periodic(rng.uniform(0, 255, (h + tpad, w + tpad)), spec.blur),
            _blur_periodic(rng.uniform(0, 255, (ch + tpad, cw + tpad)), spec.blur_uv),
            _blur_periodic(rng.uniform(0, 255, (ch + tpad, cw + tpad)), spec.blur_uv),
        ]
        n = spec.rects
        lo, hi = spec.rect_size
        self.rw = rng.integers(lo, hi + 1, n)
        self.rh = rng.integers(lo, hi + 1, n)
        self.rx = rng.integers(-lo // 2, w - lo // 2, n)
        self.ry = rng.integers(-lo // 2, h - lo // 2, n)
        self.vx = rng.integers(-4, 5, n)
        self.vy = rng.integers(-4, 5, n)
        self.val = rng.integers(30, 221, (3, n))
        self.t0 = 0

    def frame(self, t, rng):
        s = self.spec
        w, h = s.width, s.height
        cw, ch = (w + 1) // 2, (h + 1) // 2
        k = t - self.t0
        planes = []
        for p in range(3):
            pw, ph = (w, h) if p == 0 else (cw, ch)
            div = 1 if p == 0 else 2
            img = _pan_sample(self.tex[p], ph, pw, s.pan[0] * k / div, s.pan[1] * k / div)
            for i in range(s.rects):
                x = int(self.rx[i] + self.vx[i] * k) // div
                y = int(self.ry[i] + self.vy[i] * k) // div
                rw, rh = int(self.rw[i]) // div, int(self.rh[i]) // div
                x0, y0, x1, y1 = max(x, 0), max(y, 0), min(x + rw, pw), min(y + rh, ph)
                if x0 < x1 and y0 < y1:
                    img[y0:y1, x0:x1] = self.val[p, i]
            img = img + rng.normal(0.0, s.noise, img.shape)
            planes.append(np.clip(np.rint(img), 0, 255).astype(np.uint8))
        return planes


def generate(spec, frames=None):
    """Yields the clip's frames as [Y, U, V] uint8 arrays (display order)."""
    n = spec.frames if frames is None else min(frames, spec.frames)
    rng = np.random.default_rng(spec.seed)
    scene = _Scene(spec, rng)
    for t in range(n):
        if spec.cut >= 0 and t == spec.cut:
            rng = np.random.default_rng(spec.seed + 1000003)
            scene = _Scene(spec, rng)
            scene.t0 = t
        yield scene.frame(t, rng)


def packed(frame):
    """Packed I420 bytes of one frame."""
    return b"".join(p.tobytes() for p in frame)


def clip_sha256(spec, frames=None):
    h = hashlib.sha256()
    for f in generate(spec, frames):
        h.update(packed(f))
    return h.hexdigest()


def write_y4m(path, spec, frames=None):
    with open(path, "wb") as f:
        f.write(f"YUV4MPEG2 W{spec.width} H{spec.height} F30:1 Ip A1:1 C420jpeg\n".encode())
        for fr in generate(spec, frames):
            f.write(b"FRAME\n")
            f.write(packed(fr))


# ---- the batching workload: 16 streams of uneven size ---------------------------------
# 4 each of 640x360, 1280x720, 1920x1080 and 2560x1440, 60 frames, every stream
# with its own seed and the 352x288 recipe scaled to its size: pan, rectangle
# sizes and rectangle count grow with the width ratio (s = width / 352); blur
# and noise stay. Each stream's quantizer is drawn from {80, 125, 170} by a
# seeded generator.
BATCH_SIZES = [(640, 360), (1280, 720), (1920, 1080), (2560, 1440)]
BATCH_QS = (80, 125, 170)


def batch_streams(frames=60, per_size=4, seed=2024):
    """[(ClipSpec, q)] of the 16-stream batching workload."""
    rng = np.random.default_rng(seed)
    out = []
    for (w, h) in BATCH_SIZES:
        s = w / 352.0
        for k in range(per_size):
            spec = ClipSpec(w, h, frames, seed=int(rng.integers(1, 1 << 30)), blur=3.0, blur_uv=5.0,
                            pan=(1.25 * s, -0.5 * s), rects=int(round(4 * s)),
                            rect_size=(int(round(24 * s)), int(round(64 * s))), noise=2.0,
                            name=f"batch_{w}x{h}_{k}")
            out.append((spec, int(rng.choice(BATCH_QS))))
    return out


def packed_clip(spec, frames=None):
    """The clip's frames as one uint8 array [frames, packed I420 bytes]."""
    return np.stack([np.frombuffer(packed(f), np.uint8) for f in generate(spec, frames)])
