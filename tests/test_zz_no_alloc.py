"""mav1cu_edge_types_noalloc, the edge-type entry point that allocates no
device memory, against the session entry point mav1cu_edge_types: the same
BlockInfo bytes for two frames coded back to back on one caller stream.

The device buffers handed to it are the test's own (torch tensors); the
entry point itself only uses its fixed scratch array. The file's name makes
pytest collect it last, so it also runs after every other GPU test."""
import ctypes

import numpy as np
import pytest

import mav1cu
import synthetic

# (width, height, tiles, seed): a plain frame, then a ragged one with tile
# columns (the left-neighbour rule stops at tile edges).
CASES = [(352, 288, 0, 71), (203, 131, 1, 72)]


def padded_source(frame, geom):
    """I420 planes in the session's layout: superblock-aligned, edge-replicated."""
    out = []
    for p, plane in enumerate(frame):
        aw, ah = geom["stride"][p], geom["plane_h"][p]
        out.append(np.pad(plane, ((0, ah - plane.shape[0]), (0, aw - plane.shape[1])), mode="edge").ravel())
    return np.concatenate(out)


def session_case(w, h, tiles, seed):
    """Key-frame analysis on a session; returns its blocks before and after
    mav1cu_edge_types, with the params and superblock table."""
    cfg = mav1cu.cli_config(w, h, q=100, tiles=tiles)
    fp, _ = mav1cu.frame_params(cfg, mav1cu.plan(cfg, 1)[0])
    frame = next(synthetic.generate(synthetic.ClipSpec(w, h, 1, seed=seed)))
    s = mav1cu.Session(w, h)
    try:
        src = padded_source(frame, s.geom)
        assert src.size == s.size("SRC")
        s.set_params(fp)
        s.upload("SRC", src)
        s.analyze()
        before = s.download("BLOCKS")
        sbs = s.download("SBS")
        s.edge_types()
        after = s.download("BLOCKS")
        s.synchronize()
    finally:
        s.close()
    return dict(geom=s.geom, params=np.frombuffer(fp.tobytes(), np.uint8).copy(), before=before, sbs=sbs, after=after)


def call(lib, params, blocks, sbs, geom, stream):
    err = ctypes.create_string_buffer(256)
    rc = lib.mav1cu_edge_types_noalloc(params.data_ptr(), blocks.data_ptr(), sbs.data_ptr(), geom["mi_rows"],
                                       geom["mi_cols"], geom["num_sbs"], stream, err, 256)
    return rc, err.value.decode()


def test_refuses_bad_sizes_before_device_work():
    lib = mav1cu.lib()
    err = ctypes.create_string_buffer(256)
    big = 1024 * 1024 // 256 + 1
    rc = lib.mav1cu_edge_types_noalloc(1, 1, 1, 256, big * 1, 1, None, err, 256)
    assert rc == -1 and b"scratch limit" in err.value
    rc = lib.mav1cu_edge_types_noalloc(None, 1, 1, 16, 16, 1, None, err, 256)
    assert rc == -1 and b"null" in err.value
    rc = lib.mav1cu_edge_types_noalloc(1, 1, 1, 0, 16, 1, None, err, 256)
    assert rc == -1 and b"non-positive" in err.value


@pytest.mark.gpu
def test_noalloc_matches_session_entry_point_two_calls_in_a_row():
    import torch

    lib = mav1cu.lib()
    cases = [session_case(*c) for c in CASES]
    # the comparison is not vacuous: some blocks get an edge bit set
    assert any(((c["after"].view(mav1cu.BLOCK_DTYPE)["interp_filter"] >> 4) & 3).any() for c in cases)

    dev = []
    for c in cases:
        dev.append(dict(params=torch.from_numpy(c["params"]).cuda(), blocks=torch.from_numpy(c["before"]).cuda(),
                        sbs=torch.from_numpy(c["sbs"]).cuda()))
    torch.cuda.synchronize()
    stream = torch.cuda.Stream()
    for c, d in zip(cases, dev):
        rc, msg = call(lib, d["params"], d["blocks"], d["sbs"], c["geom"], stream.cuda_stream)
        assert rc == 0, msg
    stream.synchronize()
    for c, d in zip(cases, dev):
        got = d["blocks"].cpu().numpy()
        assert np.array_equal(got, c["after"])

    # the calls allocate nothing: after the warm-up above, further calls on
    # the same stream leave the device's free memory as it was
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        for c, d in zip(cases, dev):
            rc, msg = call(lib, d["params"], d["blocks"], d["sbs"], c["geom"], stream.cuda_stream)
            assert rc == 0, msg
    stream.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
