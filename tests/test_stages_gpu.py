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
