"""GPU parity: every CUDA stage against the reference's scalar CPU path
(the oracle) on the same seeded inputs, stage by stage and chained.
Bit-exact: every compared value must be equal."""
import pytest

import mav1cu
import oracle
import parity
import synthetic

pytestmark = pytest.mark.gpu

CASES = {
    # turbo (the 1080p benchmark's tool set) on the 352x288 clip: key, ALTREF and leaf frames
    "c0_turbo": (synthetic.CONFIGS["c0_352x288"], 7, dict(q=125, turbo=1, keyint=30, tiles=0)),
    # the full tool set (the 4K configuration's flags) on an odd-sized clip: tx type search,
    # tx_depth, dual filter, angle deltas, rectangular / A-B / 4-way partitions, loop restoration
    "full_203x131": (synthetic.ClipSpec(203, 131, 6, seed=11, rects=3, rect_size=(16, 48)), 6,
                     dict(q=90, altref=4, golden=1, tiles=1, me_range=64)),
    # low-delay with GOLDEN, lr_test forcing Wiener / self-guided units, odd size, q 200
    "lowdelay_lrtest": (synthetic.ClipSpec(150, 102, 5, seed=12, rects=2, rect_size=(16, 40)), 5,
                        dict(q=200, golden=1, keyint=4, lr_test=1)),
    # lossless (q 0: Walsh-Hadamard 4x4 transforms everywhere)
    "lossless": (synthetic.ClipSpec(96, 64, 3, seed=13, rects=1, rect_size=(16, 32)), 3, dict(q=0, fast=1)),
    # turbo with several tile columns at a wider size
    "turbo_tiles": (synthetic.ClipSpec(640, 360, 5, seed=14, pan=(2.5, 1.0), rects=6, rect_size=(32, 128)), 5,
                    dict(q=170, turbo=1, keyint=60, tiles=2)),
}


@pytest.fixture(scope="module", params=sorted(CASES))
def traced(request):
    if not oracle.available():
        pytest.skip("oracle library not built")
    spec, n, flags = CASES[request.param]
    tr, cfg, frames, packets, recons = parity.trace_clip(spec, n, **flags)
    sess = mav1cu.Session(spec.width, spec.height)
    yield sess, tr, cfg
    sess.close()


@pytest.mark.parametrize("stage", parity.STAGES)
def test_stage(traced, stage):
    sess, tr, cfg = traced
    bad = []
    for k, fr in enumerate(tr.frames):
        out = getattr(parity.FrameCheck(sess, tr, cfg, fr), stage)()
        if any(out.values()):
            bad.append((k, fr["state"]["frame_kind"], out))
    assert not bad, f"{stage} mismatches (frame, kind, counts): {bad}"
