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


PLANNER_DTYPE = np.dtype([(n, "<i4") for n in ["in_disp", "inq_n", "key_disp", "anchor_slot", "ld_order_hint",
                                                 "ld_last_id", "ld_gold_id"]] + [("pad", "<i4", (9,))])


@pytest.mark.parametrize("flags,n", [(dict(turbo=1, keyint=60), 120), (dict(altref=8, leaf=1), 37),
                                     (dict(altref=4, golden=1), 23), (dict(golden=1, keyint=4), 11),
                                     (dict(turbo=1, keyint=8), 9), (dict(altref=16, golden=1), 32),
                                     (dict(q=90, nonref=1), 10)])
def test_incremental_plan_equals_whole_clip(flags, n):
    """mav1cu_plan_frames fed one frame at a time, then flushed (the queue
    API's mav1_send_frame sequence), plans the same jobs in the same order as
    mav1cu_plan over the whole clip."""
    import ctypes
    L = mav1cu.lib()
    L.mav1cu_plan_frames.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                     ctypes.c_int]
    nonref = flags.pop("nonref", 0)
    cfg = mav1cu.cli_config(352, 288, **flags)
    cfg[0]["nonref_odd"] = nonref
    whole = [tuple(j) for j in mav1cu.plan(cfg, n)]
    state = np.zeros(1, PLANNER_DTYPE)
    buf = np.zeros(64, mav1cu.JOB_DTYPE)
    got = []
    for f in range(n + 1):
        k = L.mav1cu_plan_frames(cfg.ctypes.data, state.ctypes.data, 1 if f < n else 0, 1 if f == n else 0,
                                 buf.ctypes.data, len(buf))
        assert k >= 0
        got += [tuple(j) for j in buf[:k]]
    assert got == whole
    assert state[0]["in_disp"] == n and state[0]["inq_n"] == 0
