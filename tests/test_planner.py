"""The product's frame driver (coding order, quantizer cascade, frame
parameters) against the oracle's: for every coded frame the FrameParams
record must be byte-identical, in the same coding order. CPU only."""
import numpy as np
import pytest

import mav1cu
import oracle
import parity
import synthetic

CASES = [
    # (clip, frames, flags)
    (synthetic.ClipSpec(352, 288, 13, seed=3), 13, dict(q=125, turbo=1, keyint=30, tiles=0)),
    (synthetic.ClipSpec(352, 288, 13, seed=3), 13, dict(q=125, turbo=1, keyint=5, tiles=0)),
    (synthetic.ClipSpec(203, 131, 11, seed=4), 11, dict(q=90, altref=8, golden=1, tiles=3, me_range=64)),
    (synthetic.ClipSpec(203, 131, 11, seed=5), 11, dict(q=60, altref=6, leaf=1, lr=0)),
    (synthetic.ClipSpec(160, 96, 9, seed=6), 9, dict(q=180, golden=1, keyint=4)),
    (synthetic.ClipSpec(160, 96, 7, seed=7), 7, dict(q=0, fast=1)),
]


@pytest.mark.skipif(not oracle.available(), reason="oracle not built")
@pytest.mark.parametrize("case", range(len(CASES)))
def test_frame_params_match_oracle(case):
    spec, n, flags = CASES[case]
    tr = oracle.Trace(stages={oracle.STAGE["PARAMS"]})
    oracle.encode(list(synthetic.generate(spec, n)), oracle.cli_config(spec.width, spec.height, **flags), trace=tr)
    cfg = mav1cu.cli_config(spec.width, spec.height, **flags)
    jobs = mav1cu.plan(cfg, n)
    assert len(jobs) == len(tr.frames)
    for k, (job, fr) in enumerate(zip(jobs, tr.frames)):
        fp, _ = mav1cu.frame_params(cfg, job)
        ref = parity.params_of(fr)
        assert np.array_equal(fp, ref), (k, job, np.flatnonzero(fp.view(np.int32) != ref.view(np.int32)))
