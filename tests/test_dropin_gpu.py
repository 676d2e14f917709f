"""The drop-in: the encoder's own driver, tile writer and LR search with the
CUDA backend behind the unchanged Backend vtable (backend_cuda.c over
libmav1cu) against the same driver with the reference CPU backend. The IVF
bitstreams, the reconstructions returned by mav1_get_recon and the
MAV1_DUMP_DEC decision dumps must be byte-identical."""
import os

import numpy as np
import pytest

import oracle
import synthetic

pytestmark = pytest.mark.gpu

CASES = {
    "c0_turbo": (synthetic.CONFIGS["c0_352x288"], 13, dict(q=125, turbo=1, keyint=30, tiles=0)),
    "full_tools": (synthetic.ClipSpec(203, 131, 7, seed=31, rects=3, rect_size=(16, 48)), 7,
                   dict(q=90, altref=4, golden=1, tiles=1, me_range=64)),
    "lowdelay_lr": (synthetic.ClipSpec(150, 102, 5, seed=32, rects=2, rect_size=(16, 40)), 5,
                    dict(q=200, golden=1, keyint=4, lr_test=1)),
    "lossless": (synthetic.ClipSpec(96, 64, 3, seed=33, rects=1, rect_size=(16, 32)), 3, dict(q=0, fast=1)),
    # the benchmark clip and flags at full size (key, ALTREF, leaf and a second key frame)
    "c1_1080p_turbo": (synthetic.CONFIGS["c1_1080p"], 9, dict(q=125, turbo=1, keyint=8, tiles=2)),
    # the 4K clip's geometry (3 tile columns) with the turbo tool set
    "c2_2160p_turbo": (synthetic.CONFIGS["c2_2160p"], 3, dict(q=125, turbo=1, tiles=3)),
}


def _encode(spec, n, flags, cuda, dump):
    frames = list(synthetic.generate(spec, n))
    os.environ["MAV1_DUMP_DEC"] = dump
    try:
        path = oracle.HYB_PATH if cuda else oracle.LIB_PATH
        cfg = oracle.cli_config(spec.width, spec.height, cpu=not cuda, **flags)
        cfg_lib = oracle.lib(path)
        return oracle.encode(frames, cfg, factory="cuda" if cuda else None, path=path)
    finally:
        del os.environ["MAV1_DUMP_DEC"]


@pytest.mark.skipif(not (oracle.available() and oracle.available(oracle.HYB_PATH)), reason="oracle not built")
@pytest.mark.parametrize("name", sorted(CASES))
def test_dropin_bitstream_identical(name, tmp_path):
    spec, n, flags = CASES[name]
    pk_cpu, rec_cpu = _encode(spec, n, flags, False, str(tmp_path / "cpu.dec"))
    pk_gpu, rec_gpu = _encode(spec, n, flags, True, str(tmp_path / "cuda.dec"))
    ivf_cpu = oracle.ivf_bytes(pk_cpu, spec.width, spec.height)
    ivf_gpu = oracle.ivf_bytes(pk_gpu, spec.width, spec.height)
    assert len(pk_cpu) == len(pk_gpu)
    assert ivf_cpu == ivf_gpu, [i for i, (a, b) in enumerate(zip(pk_cpu, pk_gpu)) if a != b]
    for a, b in zip(rec_cpu, rec_gpu):
        for pa, pb in zip(a, b):
            assert np.array_equal(pa, pb)
    assert (tmp_path / "cpu.dec").read_bytes() == (tmp_path / "cuda.dec").read_bytes()


@pytest.mark.skipif(not (oracle.available() and oracle.available(oracle.HYB_PATH)), reason="oracle not built")
def test_dropin_full_tools_2160p_matches_golden(tmp_path):
    """The benchmark spec's full-tool configuration at full size (3840x2160,
    -q 90, tx search, tx depth, switchable / dual filter, CDEF, loop
    restoration, --altref 16 --golden --tiles 3, ME range 64; its first 3
    frames) through the drop-in, against SHA-256 hashes of the oracle's IVF
    bitstream, reconstructions and decision dump for the same frames
    (tests/golden/dropin_hashes.json, written by tests/golden/make_golden.py
    --large: the oracle needs minutes per frame at this size)."""
    import hashlib
    import importlib.util
    import json
    here = os.path.dirname(os.path.abspath(__file__))
    spec_ = importlib.util.spec_from_file_location("make_golden", os.path.join(here, "golden", "make_golden.py"))
    mg = importlib.util.module_from_spec(spec_)
    spec_.loader.exec_module(mg)
    name = "c2_2160p_full_3f"
    want = json.load(open(os.path.join(here, "golden", "dropin_hashes.json")))[name]
    spec, frames, flags = mg.large_frames(name)
    assert mg.frames_sha256(frames) == want["frames"]
    dump = str(tmp_path / "cuda.dec")
    packets, recons = _encode(spec, len(frames), flags, True, dump)
    h = lambda b: hashlib.sha256(b).hexdigest()
    assert len(packets) == want["packets"]
    assert h(oracle.ivf_bytes(packets, spec.width, spec.height)) == want["ivf"]
    assert h(b"".join(p.tobytes() for r in recons for p in r)) == want["recon"]
    assert h(open(dump, "rb").read()) == want["dump"]



@pytest.mark.skipif(not (oracle.available() and oracle.available(oracle.HYB_PATH)), reason="oracle not built")
def test_dropin_throughput_1080p():
    """What an unchanged mav1.h caller gets through the drop-in (the
    reference's own serial driver with backend_cuda.c behind the vtable):
    the benchmark clip's first 60 frames (1920x1080, --turbo -q 125 --keyint
    60 --tiles 2), timed by wall clock, against the encoder API library on
    the same frames. Every hook of the drop-in copies the encoder's full host
    buffers to and from the device and synchronises, so it is far slower
    than the API library; the printed figures show by how much. Both
    bitstreams equal the reference CPU path's."""
    import time

    import mav1api
    import mav1cu

    spec, n = synthetic.CONFIGS["c1_1080p"], 60
    flags = dict(q=125, turbo=1, keyint=60, tiles=2)
    frames = list(synthetic.generate(spec, n))
    pk_cpu, _ = oracle.encode(frames, oracle.cli_config(spec.width, spec.height, cpu=True, **flags))
    cfg_hyb = oracle.cli_config(spec.width, spec.height, cpu=False, **flags)
    oracle.encode(frames[:2], cfg_hyb, factory="cuda", path=oracle.HYB_PATH)  # warm-up
    t0 = time.perf_counter()
    pk_hyb, _ = oracle.encode(frames, cfg_hyb, factory="cuda", path=oracle.HYB_PATH)
    t_hyb = time.perf_counter() - t0
    packed = [np.frombuffer(synthetic.packed(f), np.uint8) for f in frames]
    cfg_api = mav1cu.cli_config(spec.width, spec.height, **flags)
    mav1api.encode(packed[:2], cfg_api, recon=False)  # warm-up
    t0 = time.perf_counter()
    pk_api, _ = mav1api.encode(packed, cfg_api, recon=True)
    t_api = time.perf_counter() - t0
    ivf = lambda pk: oracle.ivf_bytes(pk, spec.width, spec.height)
    assert ivf(pk_hyb) == ivf(pk_cpu)
    assert mav1api.ivf_bytes(pk_api, spec.width, spec.height) == ivf(pk_cpu)
    print(f"\ndrop-in (reference driver + backend_cuda.c): {n / t_hyb:.1f} fps; "
          f"encoder API library (libmav1.so), one encoder: {n / t_api:.1f} fps")
