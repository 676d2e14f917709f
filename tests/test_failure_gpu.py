"""Failure detection without a device fault: a dependency that is never
released makes the intra reconstruction's bounded waits give up; the launch
returns, the session reports MAV1CU_ERR_DEVICE, and the context stays usable
(another session codes the same frame correctly afterwards). Nothing here
traps, faults or hangs the GPU: the wait limit is a few thousand polls."""
import time

import numpy as np
import pytest

import mav1cu
import synthetic

pytestmark = pytest.mark.gpu


def padded_source(frame, geom):
    out = []
    for p, plane in enumerate(frame):
        aw, ah = geom["stride"][p], geom["plane_h"][p]
        out.append(np.pad(plane, ((0, ah - plane.shape[0]), (0, aw - plane.shape[1])), mode="edge").ravel())
    return np.concatenate(out)


def key_frame_session(w, h, seed):
    cfg = mav1cu.cli_config(w, h, q=100, turbo=1)
    fp, _ = mav1cu.frame_params(cfg, mav1cu.plan(cfg, 1)[0])
    frame = next(synthetic.generate(synthetic.ClipSpec(w, h, 1, seed=seed)))
    s = mav1cu.Session(w, h)
    s.set_params(fp)
    s.upload("SRC", padded_source(frame, s.geom))
    return s


def test_never_released_dependency_reports_device_error():
    w, h = 160, 96
    bad = key_frame_session(w, h, 81)
    try:
        # block 0 (the first block of the first superblock) is never released:
        # every other intra block depends on it, so every worker waits
        rc = bad.lib.mav1cu_debug_recon_fault(bad.h, 0, 4096)
        assert rc == 0
        t0 = time.perf_counter()
        bad.frame_core()
        with pytest.raises(mav1cu.Mav1cuError, match="gave up"):
            bad.synchronize()
        assert time.perf_counter() - t0 < 10.0
        # sticky: the session stays in error
        with pytest.raises(mav1cu.Mav1cuError):
            bad.synchronize()
    finally:
        bad.close()
    # the context is usable: the same frame codes on a fresh session, twice
    # alike (bit-exactness against the oracle is covered by the stage tests)
    outs = []
    for _ in range(2):
        good = key_frame_session(w, h, 81)
        try:
            good.frame_core()
            good.synchronize()
            outs.append(good.download("REC"))
        finally:
            good.close()
    assert np.array_equal(outs[0], outs[1])


def test_fault_hook_rejects_bad_arguments():
    s = key_frame_session(64, 64, 82)
    try:
        assert s.lib.mav1cu_debug_recon_fault(s.h, -1, 100) == -1
    finally:
        s.close()
