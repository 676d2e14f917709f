#!/usr/bin/env python3
"""Writes tests/golden/oracle_hashes.json: SHA-256 of the oracle's output
(IVF bitstream, shown reconstructions, MAV1_DUMP_DEC decision dump) for
seeded synthetic clips, plus the hash of the clips themselves. Run on a
machine with the oracle built (make -C oracle); the fixture pins the oracle
(the reference's scalar CPU path) so later runs detect any change in it."""
import hashlib
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "mav1-encoder_b200"), os.path.join(ROOT, "oracle")]

import oracle  # noqa: E402
import synthetic  # noqa: E402

CASES = {
    "c0_turbo_q125": (dict(width=352, height=288, frames=30, seed=1), dict(q=125, turbo=1, keyint=30, tiles=0)),
    "full_203x131": (dict(width=203, height=131, frames=9, seed=41, rects=3, rect_size=(16, 48)),
                     dict(q=90, altref=4, golden=1, tiles=1, me_range=64)),
    "lowdelay_lr_150x102": (dict(width=150, height=102, frames=6, seed=42, rects=2, rect_size=(16, 40)),
                            dict(q=200, golden=1, keyint=4, lr_test=1)),
    "lossless_96x64": (dict(width=96, height=64, frames=3, seed=43, rects=1, rect_size=(16, 32)), dict(q=0, fast=1)),
    # the benchmark workload: the whole 120-frame 1080p clip with its flags
    "c1_1080p_turbo_120": (dict(width=1920, height=1080, frames=120, seed=1, pan=(2.5, 1.0), rects=12,
                                rect_size=(64, 256)), dict(q=125, turbo=1, keyint=60, tiles=2)),
}


def run(name):
    spec_kw, flags = CASES[name]
    spec = synthetic.ClipSpec(**spec_kw)
    frames = list(synthetic.generate(spec))
    with tempfile.TemporaryDirectory() as d:
        dump = os.path.join(d, "dec")
        os.environ["MAV1_DUMP_DEC"] = dump
        try:
            packets, recons = oracle.encode(frames, oracle.cli_config(spec.width, spec.height, **flags))
        finally:
            del os.environ["MAV1_DUMP_DEC"]
        dec = open(dump, "rb").read()
    h = lambda b: hashlib.sha256(b).hexdigest()
    return {
        "clip": synthetic.clip_sha256(spec),
        "ivf": h(oracle.ivf_bytes(packets, spec.width, spec.height)),
        "recon": h(b"".join(p.tobytes() for r in recons for p in r)),
        "dump": h(dec),
        "packets": len(packets),
        # per temporal unit: the first 16 hex digits of the SHA-256 of its
        # bytes and of its shown reconstruction (locates a difference)
        "packet_sha16": [h(p)[:16] for p in packets],
        "recon_sha16": [h(b"".join(p.tobytes() for p in r))[:16] for r in recons],
    }


# Full-size cases, too slow for the oracle inside a test (minutes of CPU
# per 4K frame with every tool on): their hashes are checked against the
# CUDA backend through the drop-in (tests/test_dropin_gpu.py). Written to
# dropin_hashes.json by `make_golden.py --large`.
LARGE_CASES = {
    # the benchmark spec's full-tool configuration (3840x2160, -q 90, tx
    # search, tx depth, switchable / dual filter, CDEF, loop restoration,
    # --altref 16 --golden --tiles 3, ME range 64): its first 3 frames
    "c2_2160p_full_3f": ("c2_2160p", 3, dict(q=90, altref=16, golden=1, tiles=3, me_range=64)),
    # the whole configuration: 32 frames, the scene cut at frame 16
    "c2_2160p_full_32f": ("c2_2160p", 32, dict(q=90, altref=16, golden=1, tiles=3, me_range=64)),
}


def large_frames(name):
    clip, n, flags = LARGE_CASES[name]
    spec = synthetic.CONFIGS[clip]
    return spec, list(synthetic.generate(spec, n)), flags


def frames_sha256(frames):
    return hashlib.sha256(b"".join(synthetic.packed(f) for f in frames)).hexdigest()


def run_large(name):
    spec, frames, flags = large_frames(name)
    with tempfile.TemporaryDirectory() as d:
        dump = os.path.join(d, "dec")
        os.environ["MAV1_DUMP_DEC"] = dump
        try:
            packets, recons = oracle.encode(frames, oracle.cli_config(spec.width, spec.height, **flags))
        finally:
            del os.environ["MAV1_DUMP_DEC"]
        dec = open(dump, "rb").read()
    h = lambda b: hashlib.sha256(b).hexdigest()
    return {
        "frames": frames_sha256(frames),
        "ivf": h(oracle.ivf_bytes(packets, spec.width, spec.height)),
        "recon": h(b"".join(p.tobytes() for r in recons for p in r)),
        "dump": h(dec),
        "packets": len(packets),
        "packet_sha16": [h(p)[:16] for p in packets],
    }


def run_batch():
    """The 16-stream batching workload (synthetic.batch_streams, --turbo with
    each stream's q): per stream the hashes of its clip, IVF bitstream and
    shown reconstructions as the oracle codes it alone."""
    h = lambda b: hashlib.sha256(b).hexdigest()
    out = {}
    for spec, q in synthetic.batch_streams():
        frames = list(synthetic.generate(spec))
        packets, recons = oracle.encode(frames, oracle.cli_config(spec.width, spec.height, q=q, turbo=1))
        out[spec.name] = {
            "clip": hashlib.sha256(b"".join(synthetic.packed(f) for f in frames)).hexdigest(),
            "q": q,
            "ivf": h(oracle.ivf_bytes(packets, spec.width, spec.height)),
            "recon": h(b"".join(p.tobytes() for r in recons for p in r)),
            "packets": len(packets),
        }
        print(spec.name, out[spec.name]["ivf"][:16], flush=True)
    return out


if __name__ == "__main__":
    if "--batch" in sys.argv:
        out = run_batch()
        json.dump(out, open(os.path.join(HERE, "batch_hashes.json"), "w"), indent=1, sort_keys=True)
    elif "--large" in sys.argv:
        # --case NAME recomputes one entry and keeps the others
        names = [sys.argv[sys.argv.index("--case") + 1]] if "--case" in sys.argv else list(LARGE_CASES)
        path = os.path.join(HERE, "dropin_hashes.json")
        out = json.load(open(path)) if os.path.exists(path) and "--case" in sys.argv else {}
        out.update({name: run_large(name) for name in names})
        json.dump(out, open(path, "w"), indent=1, sort_keys=True)
    else:
        # --case NAME recomputes one entry and keeps the others
        names = [sys.argv[sys.argv.index("--case") + 1]] if "--case" in sys.argv else list(CASES)
        path = os.path.join(HERE, "oracle_hashes.json")
        out = json.load(open(path)) if os.path.exists(path) and "--case" in sys.argv else {}
        out.update({name: run(name) for name in names})
        json.dump(out, open(path, "w"), indent=1, sort_keys=True)
    print(json.dumps(out, indent=1))
