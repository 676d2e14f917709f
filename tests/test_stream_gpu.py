"""The device-resident stream (frame planning, source load, every stage,
slot refresh, two concurrent frame engines) against the oracle over whole
clips: every frame's writer inputs (blocks, superblock table, coefficients,
CDEF choices) and reconstruction, in coding order, bit-exact."""
import pytest

import oracle
import parity
import synthetic

pytestmark = pytest.mark.gpu

CASES = {
    "c0_turbo_13": (synthetic.CONFIGS["c0_352x288"], 13, dict(q=125, turbo=1, keyint=30, tiles=0)),
    "turbo_keyint5": (synthetic.ClipSpec(320, 200, 12, seed=21, rects=5, rect_size=(20, 80)), 12,
                      dict(q=80, turbo=1, keyint=5, tiles=1)),
    "lowdelay_golden": (synthetic.ClipSpec(176, 144, 8, seed=22, rects=3), 8,
                        dict(q=150, golden=1, keyint=6, lr=0, tiles=1)),
}


class _WriterTrace(oracle.Trace):
    """Only what the stream comparison reads (keeps a 1080p trace small)."""
    CAPTURE = {
        oracle.STAGE["PARAMS"]: ["PARAMS"],
        oracle.STAGE["ANALYZE"]: ["SBS"],
        oracle.STAGE["RECON"]: ["BLOCKS", "COEFS"],
        oracle.STAGE["CDEFSEL"]: ["CDEF_CHOICE"],
        oracle.STAGE["DONE"]: ["REC"],
    }


@pytest.mark.skipif(not oracle.available(), reason="oracle not built")
def test_stream_matches_oracle_1080p():
    """The benchmark's clip and flags at full size through the device stream:
    key, ALTREF and leaf frames and a second key frame (keyint 8)."""
    spec, n = synthetic.CONFIGS["c1_1080p"], 9
    flags = dict(q=125, turbo=1, keyint=8, tiles=2)
    frames = list(synthetic.generate(spec, n))
    tr = _WriterTrace()
    oracle.encode(frames, oracle.cli_config(spec.width, spec.height, **flags), trace=tr)
    res = parity.stream_vs_oracle(tr, frames, flags, spec)
    bad = [(k, o) for k, o in res if any(o.values())]
    assert not bad, bad


@pytest.mark.skipif(not oracle.available(), reason="oracle not built")
@pytest.mark.parametrize("name", sorted(CASES))
def test_stream_matches_oracle(name):
    spec, n, flags = CASES[name]
    tr, cfg, frames, packets, recons = parity.trace_clip(spec, n, **flags)
    res = parity.stream_vs_oracle(tr, frames, flags, spec)
    bad = [(k, o) for k, o in res if any(o.values())]
    assert not bad, bad
