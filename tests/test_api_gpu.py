"""The mav1 encoder API (libmav1.so: src/mav1.h of the reference, unchanged)
on the B200 backend, end to end: device stream, host entropy pool, temporal
units. Its IVF bitstreams, the reconstructions mav1_get_recon returns and
the MAV1_DUMP_DEC decision records must equal the oracle's (the reference's
scalar CPU path) byte for byte.

Also: the reference's own command-line encoder (tools/mav1enc.c, unchanged)
linked against libmav1.so against the oracle's build of the same CLI, and
the benchmark workload (the whole 120-frame 1080p clip) coded the way
bench.py times it, against committed hashes of the oracle's output."""
import hashlib
import json
import os
import subprocess
import threading

import numpy as np
import pytest

import mav1api
import mav1cu
import oracle
import synthetic

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "oracle_hashes.json")))

# clips and CLI flags (tools/mav1enc.c) of the cases
CASES = {
    "c0_turbo": (synthetic.CONFIGS["c0_352x288"], 13, dict(q=125, turbo=1, keyint=30, tiles=0)),
    # ALTREF 4 without the turbo savings: pyramid-free mini-GOPs, tx search, tx depth, switchable filters
    "full_tools_nolr": (synthetic.ClipSpec(203, 131, 9, seed=31, rects=3, rect_size=(16, 48)), 9,
                        dict(q=90, altref=4, golden=1, tiles=1, me_range=64, lr=0)),
    # pyramid leaf frames (altref 8 + leaf): hidden middle frames and nested show_existing
    "pyramid_leaf": (synthetic.ClipSpec(160, 96, 17, seed=34, rects=2), 17, dict(q=110, altref=8, leaf=1, lr=0)),
    # the low-delay path (mav1_encode): GOLDEN every 4th frame, key frames every 4
    "lowdelay": (synthetic.ClipSpec(150, 102, 6, seed=32, rects=2, rect_size=(16, 40)), 6,
                 dict(q=200, golden=1, keyint=4, lr=0)),
    "lossless": (synthetic.ClipSpec(96, 64, 3, seed=33, rects=1, rect_size=(16, 32)), 3, dict(q=0, fast=1)),
    # the full tool set of the 4K configuration (loop restoration included) on an odd-sized clip
    "full_tools": (synthetic.ClipSpec(203, 131, 9, seed=31, rects=3, rect_size=(16, 48)), 9,
                   dict(q=90, altref=4, golden=1, tiles=1, me_range=64)),
    # low delay with lr_test (Wiener and self-guided units forced), q 200
    "lowdelay_lrtest": (synthetic.ClipSpec(150, 102, 6, seed=32, rects=2, rect_size=(16, 40)), 6,
                        dict(q=200, golden=1, keyint=4, lr_test=1)),
    # loop restoration on a wider frame with several tile columns and ALTREF 16
    "lr_altref16": (synthetic.ClipSpec(640, 360, 20, seed=35, rects=5, rect_size=(32, 96), cut=12), 20,
                    dict(q=110, altref=16, tiles=2)),
    # the benchmark clip and flags (key, ALTREF, leaf and a second key frame)
    "c1_1080p_turbo": (synthetic.CONFIGS["c1_1080p"], 9, dict(q=125, turbo=1, keyint=8, tiles=2)),
}


def _h(b):
    return hashlib.sha256(b).hexdigest()


def _oracle(spec, frames, flags, dump):
    os.environ["MAV1_DUMP_DEC"] = dump
    try:
        return oracle.encode(frames, oracle.cli_config(spec.width, spec.height, **flags))
    finally:
        del os.environ["MAV1_DUMP_DEC"]


def _ours(spec, frames, flags, dump):
    os.environ["MAV1_DUMP_DEC"] = dump
    try:
        cfg = mav1cu.cli_config(spec.width, spec.height, **flags)
        return mav1api.encode([synthetic.packed(f) for f in frames], cfg)
    finally:
        del os.environ["MAV1_DUMP_DEC"]


@pytest.mark.skipif(not oracle.available(), reason="oracle not built")
@pytest.mark.parametrize("name", sorted(CASES))
def test_api_matches_oracle(name, tmp_path):
    spec, n, flags = CASES[name]
    frames = list(synthetic.generate(spec, n))
    pk_ref, rec_ref = _oracle(spec, frames, flags, str(tmp_path / "ref.dec"))
    pk, rec = _ours(spec, frames, flags, str(tmp_path / "ours.dec"))
    assert len(pk) == len(pk_ref)
    assert [i for i, (a, b) in enumerate(zip(pk, pk_ref)) if a != b] == []
    for a, b in zip(rec, rec_ref):
        for pa, pb in zip(a, b):
            assert np.array_equal(pa, pb)
    assert (tmp_path / "ours.dec").read_bytes() == (tmp_path / "ref.dec").read_bytes()


@pytest.mark.skipif(not oracle.available(), reason="oracle not built")
def test_reference_cli_on_this_backend(tmp_path):
    """tools/mav1enc.c, built unchanged against libmav1.so, writes the same
    IVF file and reconstruction (-r) as the oracle's build of the same CLI
    with --cpu."""
    spec = synthetic.ClipSpec(352, 288, 12, seed=5, rects=4)
    y4m = tmp_path / "in.y4m"
    synthetic.write_y4m(str(y4m), spec)
    flags = ["--turbo", "-q", "125", "--keyint", "30", "--tiles", "0"]
    ref_cli = os.path.join(os.path.dirname(oracle.LIB_PATH), "mav1enc")
    subprocess.run([ref_cli, "-i", str(y4m), "-o", str(tmp_path / "ref.ivf"), "-r", str(tmp_path / "ref.y4m"),
                    "--cpu"] + flags, check=True, capture_output=True)
    subprocess.run([mav1api.CLI_PATH, "-i", str(y4m), "-o", str(tmp_path / "ours.ivf"), "-r",
                    str(tmp_path / "ours.y4m")] + flags, check=True, capture_output=True)
    assert (tmp_path / "ours.ivf").read_bytes() == (tmp_path / "ref.ivf").read_bytes()
    assert (tmp_path / "ours.y4m").read_bytes() == (tmp_path / "ref.y4m").read_bytes()


def test_cpu_backend_refused():
    spec = synthetic.ClipSpec(64, 64, 1)
    cfg = mav1cu.cli_config(64, 64, q=100)
    cfg[0]["use_metal"] = 0
    with pytest.raises(mav1api.Mav1Error, match="GPU only"):
        mav1api.Encoder(cfg)


def split_at_keys(frames, keyint):
    """Runs of frames that start at a key frame (display index % keyint == 0):
    closed GOPs that independent encoders code to the same bitstream as one
    encoder (a key frame refreshes every reference slot)."""
    return [frames[i:i + keyint] for i in range(0, len(frames), keyint)]


def encode_gop_parallel(frames, cfg, keyint):
    """The benchmark's end-to-end schedule: one encoder per closed GOP, all
    running concurrently from their own host threads, each fed packed I420
    frames from host memory; the temporal units concatenated in GOP order."""
    gops = split_at_keys(frames, keyint)
    out = [None] * len(gops)

    def run(i):
        out[i] = mav1api.encode(gops[i], cfg)

    th = [threading.Thread(target=run, args=(i,)) for i in range(len(gops))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    packets = [p for pk, _ in out for p in pk]
    recons = [r for _, rc in out for r in rc]
    return packets, recons


def test_benchmark_clip_matches_golden():
    """The benchmark workload (1920x1080, 120 frames, --turbo -q 125 --keyint
    60 --tiles 2) through the API in bench.py's end-to-end schedule (two
    concurrent encoders, one per closed GOP), against the oracle's hashes of
    the whole clip coded by one encoder (tests/golden/oracle_hashes.json)."""
    want = GOLDEN["c1_1080p_turbo_120"]
    spec = synthetic.CONFIGS["c1_1080p"]
    frames = [synthetic.packed(f) for f in synthetic.generate(spec)]
    assert hashlib.sha256(b"".join(frames)).hexdigest() == want["clip"]
    cfg = mav1cu.cli_config(spec.width, spec.height, q=125, turbo=1, keyint=60, tiles=2)
    packets, recons = encode_gop_parallel(frames, cfg, 60)
    got = [_h(p)[:16] for p in packets]
    assert len(got) == want["packets"]
    assert [i for i, (a, b) in enumerate(zip(got, want["packet_sha16"])) if a != b] == []
    assert _h(mav1api.ivf_bytes(packets, spec.width, spec.height)) == want["ivf"]
    assert _h(b"".join(p.tobytes() for r in recons for p in r)) == want["recon"]


def _mg():
    import importlib.util
    spec_ = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec_)
    spec_.loader.exec_module(mg)
    return mg


@pytest.mark.parametrize("name", ["c2_2160p_full_3f", "c2_2160p_full_32f"])
def test_api_full_tools_2160p_matches_golden(name, tmp_path):
    """The benchmark spec's full-tool configuration at full size (3840x2160,
    -q 90, tx search, tx depth, switchable / dual filter, CDEF, loop
    restoration searched on the device, --altref 16 --golden --tiles 3, ME
    range 64; the first 3 frames, and all 32 with the scene cut at frame 16)
    through the API, against the oracle's hashes (tests/golden/
    dropin_hashes.json, written by make_golden.py --large)."""
    hashes = json.load(open(os.path.join(HERE, "golden", "dropin_hashes.json")))
    if name not in hashes:
        pytest.skip(f"no golden hashes for {name}")
    want = hashes[name]
    mg = _mg()
    spec, frames, flags = mg.large_frames(name)
    assert mg.frames_sha256(frames) == want["frames"]
    dump = str(tmp_path / "ours.dec")
    packets, recons = _ours(spec, frames, flags, dump)
    assert len(packets) == want["packets"]
    if "packet_sha16" in want:
        got = [_h(p)[:16] for p in packets]
        assert [i for i, (a, b) in enumerate(zip(got, want["packet_sha16"])) if a != b] == []
    assert _h(mav1api.ivf_bytes(packets, spec.width, spec.height)) == want["ivf"]
    assert _h(b"".join(p.tobytes() for r in recons for p in r)) == want["recon"]
    assert _h(open(dump, "rb").read()) == want["dump"]
