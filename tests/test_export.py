"""The compact export of the writer inputs (mav1cu_export).

CPU: the packed form is read by the reference's own host steps as it stands.
The oracle encoder runs each clip twice; in the second run, right after recon,
its BLOCKS / SBS / COEFS buffers are replaced by the packed sections (the
rest of each buffer filled with poison), and the bitstream must not change.

GPU: the image the device writes into mapped host memory equals the packing
of the dense buffers, frame by frame, through the device stream, and its
reconstruction section equals the visible samples of REC; a device memory
image equals a host one; bad images are refused."""
import ctypes

import numpy as np
import pytest

import mav1cu
import oracle
import parity
import synthetic
from mav1cu import BLOCK_DTYPE, PARAMS_DTYPE, SB_DTYPE

CPU_CASES = {
    "turbo": (synthetic.ClipSpec(200, 136, 5, seed=61, rects=3, rect_size=(16, 48)),
              dict(q=125, turbo=1, keyint=4, tiles=1)),
    "full_tools": (synthetic.ClipSpec(203, 131, 4, seed=31, rects=3, rect_size=(16, 48)),
                   dict(q=90, altref=4, golden=1, tiles=1, me_range=64)),
    "lowdelay_lr": (synthetic.ClipSpec(150, 102, 3, seed=32, rects=2, rect_size=(16, 40)),
                    dict(q=200, golden=1, keyint=4, lr_test=1)),
    "lossless": (synthetic.ClipSpec(96, 64, 2, seed=33, rects=1, rect_size=(16, 32)), dict(q=0, fast=1)),
}


class PackAfterRecon:
    """Oracle stage hook: after recon, the encoder's writer inputs become the
    packed sections; every byte past them is poison."""

    def __init__(self):
        self.frames = []

        def hook(user, stage, e):
            if stage != oracle.STAGE["RECON"]:
                return
            g = oracle.geometry(e)
            nsb = g["num_sbs"]
            p = oracle.snapshot(e, "PARAMS")[: PARAMS_DTYPE.itemsize].view(PARAMS_DTYPE)[0]
            blocks = oracle.snapshot(e, "BLOCKS", nsb * 64 * BLOCK_DTYPE.itemsize).view(BLOCK_DTYPE)
            sbs = oracle.snapshot(e, "SBS")[: nsb * SB_DTYPE.itemsize].view(SB_DTYPE)
            coefs = oracle.snapshot(e, "COEFS", nsb * 6144 * 4).view(np.int32)
            packed = parity.pack_writer_inputs(blocks, sbs, coefs, np.zeros(nsb, np.int8), p)
            dense = int(coefs.size)
            T = parity.spec_tables()
            tx64 = 0  # coded planes of 64-point transforms (their runs end at the 32 x 32 adjusted area)
            for b in packed["blocks"]:
                for pl in range(3):
                    if b["eob"][pl]:
                        tx, _ = parity.tx_layout(b, pl, p)
                        tx64 += max(T["Tx_Width"][tx], T["Tx_Height"][tx]) == 64
            self.frames.append(dict(blocks=len(packed["blocks"]), levels=len(packed["levels"]), dense=dense,
                                    zero_run=packed["zero_run"], tx64=int(tx64),
                                    coded=int(sum(b["eob"].any() for b in packed["blocks"]))))
            for name, data, poison in (("SBS", packed["sbs"], 0xA5), ("BLOCKS", packed["blocks"], 0xA5),
                                       ("COEFS", packed["levels"], 0x3F)):
                ptr, size = oracle.buf(e, name)
                raw = np.ascontiguousarray(data).view(np.uint8)
                assert raw.nbytes <= size, (name, raw.nbytes, size)
                ctypes.memset(ptr + raw.nbytes, poison, size - raw.nbytes)
                ctypes.memmove(ptr, raw.ctypes.data, raw.nbytes)

        self.cb = oracle.HOOK(hook)


pytestmark_oracle = pytest.mark.skipif(not oracle.available(), reason="oracle not built")


@pytestmark_oracle
@pytest.mark.parametrize("name", sorted(CPU_CASES))
def test_packed_inputs_give_the_same_bitstream(name):
    spec, flags = CPU_CASES[name]
    frames = list(synthetic.generate(spec))
    cfg = oracle.cli_config(spec.width, spec.height, **flags)
    plain, _ = oracle.encode(frames, cfg)
    hook = PackAfterRecon()
    packed, _ = oracle.encode(frames, oracle.cli_config(spec.width, spec.height, **flags), trace=hook)
    assert hook.frames, "the recon hook never ran"
    assert oracle.ivf_bytes(packed, spec.width, spec.height) == oracle.ivf_bytes(plain, spec.width, spec.height)
    for f in hook.frames:
        assert f["levels"] <= f["dense"]
    # the cases exercise both kinds of plane: coded blocks, and zero planes
    # of coded blocks aliased to the zero run
    assert any(f["coded"] for f in hook.frames)
    if name != "lossless":
        assert any(f["zero_run"] for f in hook.frames)
    if name in ("turbo", "full_tools"):
        assert any(f["tx64"] for f in hook.frames)


def test_packer_on_a_constructed_superblock():
    """Hand-made superblock: a skipped block, a block with only luma coded,
    and a block that lies partly outside the frame."""
    p = np.zeros(1, PARAMS_DTYPE)[0]
    p["mi_cols"], p["mi_rows"], p["lossless"] = 12, 16, 0
    T = parity.spec_tables()
    blocks = np.zeros(64, BLOCK_DTYPE)
    sbs = np.zeros(1, SB_DTYPE)
    sbs[0]["num_blocks"] = 3
    # 32x32 at (0,0): skipped
    blocks[0]["bsize"], blocks[0]["coef_off"] = 9, (0, 1024, 1280)
    # 32x32 at (0,8) (mi units): only luma coded; columns 48.. are outside the 48-wide frame
    blocks[1]["bsize"], blocks[1]["mi_col"], blocks[1]["is_inter"] = 9, 8, 1
    blocks[1]["eob"], blocks[1]["coef_off"] = (1, 0, 0), (1536, 2560, 2816)
    # 16x16 at (8,0): all planes coded
    blocks[2]["bsize"], blocks[2]["mi_row"], blocks[2]["is_inter"] = 6, 8, 1
    blocks[2]["eob"], blocks[2]["coef_off"] = (1, 1, 1), (3072, 3328, 3392)
    coefs = np.arange(6144, dtype=np.int32) + 1
    out = parity.pack_writer_inputs(blocks, sbs, coefs, np.array([3], np.int8), p)
    # block 1: 32x32 luma transform, fully inside (x 32..63 starts at 32 < 48): 1024 levels;
    # its chroma planes (16x16, start 16 < 24) are zero: run of 256
    assert T["Max_Tx_Size_Rect"][9] == 3
    assert out["zero_run"] == 256
    assert list(out["blocks"]["coef_off"][0]) == [0, 0, 0]
    assert list(out["blocks"]["coef_off"][1]) == [256, 0, 0]
    assert list(out["blocks"]["coef_off"][2]) == [256 + 1024, 256 + 1024 + 256, 256 + 1024 + 256 + 64]
    assert len(out["levels"]) == 256 + 1024 + 256 + 64 + 64
    assert np.array_equal(out["levels"][256:1280], coefs[1536:2560])
    assert np.array_equal(out["levels"][1280:1536], coefs[3072:3328])
    assert not out["levels"][:256].any()
    assert out["sbs"][0]["first_block"] == 0 and out["cdef"][0] == 3


# ---- GPU --------------------------------------------------------------------------


def _pinned(n):
    import torch
    return torch.empty(n, dtype=torch.uint8).pin_memory()


@pytest.mark.gpu
@pytest.mark.parametrize("name,spec,flags", [
    ("turbo_keyint5", synthetic.ClipSpec(200, 136, 6, seed=62, rects=3, rect_size=(16, 48)),
     dict(q=125, turbo=1, keyint=5, tiles=1)),
    ("lowdelay_golden", synthetic.ClipSpec(150, 102, 4, seed=63, rects=2, rect_size=(16, 40)),
     dict(q=200, golden=1, keyint=4, lr=0)),
    ("1080p_turbo", synthetic.CONFIGS["c1_1080p"], dict(q=125, turbo=1, keyint=60, tiles=2)),
])
def test_stream_export_matches_packing(name, spec, flags):
    import torch
    nframes = 4 if name == "1080p_turbo" else spec.frames
    frames = [np.ascontiguousarray(np.frombuffer(synthetic.packed(f), np.uint8))
              for f in synthetic.generate(spec, nframes)]
    cfg = mav1cu.cli_config(spec.width, spec.height, **flags)
    jobs = mav1cu.plan(cfg, nframes)
    st = mav1cu.Stream(cfg)
    dframes = [torch.from_numpy(f).cuda() for f in frames]
    try:
        cap = st.session.export_capacity()
        image = _pinned(cap)
        for k, job in enumerate(jobs):
            sess = st.encode(job, dframes[job["disp"]].data_ptr(), True)
            sess.export(image.data_ptr(), cap, rec=not job["hidden"])
            st.synchronize()
            img = image.numpy().copy()
            h = img[:mav1cu.EXPORT_HEADER_DTYPE.itemsize].view(mav1cu.EXPORT_HEADER_DTYPE)[0]
            assert h["status"] == 0 and h["num_sbs"] == sess.geom["num_sbs"]
            nsb = sess.geom["num_sbs"]
            blocks = sess.download("BLOCKS").view(BLOCK_DTYPE)
            sbs = sess.download("SBS").view(SB_DTYPE)[:nsb]
            coefs = sess.download("COEFS", np.int32)
            cdef = sess.download("CDEF_CHOICE", np.int8, count=nsb)
            p = sess.download("PARAMS", count=PARAMS_DTYPE.itemsize).view(PARAMS_DTYPE)[0]
            bad = {k_: v for k_, v in parity.export_vs_packed(img, blocks, sbs, coefs, cdef, p).items() if v}
            assert not bad, (k, bad)
            rec = mav1cu.export_sections(img)[5]
            if job["hidden"]:
                assert rec is None
            else:
                # mav1_get_recon's planes: the visible samples of REC
                assert np.array_equal(rec, parity.visible(sess.download("REC"), sess.geom)), k
            assert h["bytes"] - h["rec_bytes"] < (nsb * (SB_DTYPE.itemsize + 64 * BLOCK_DTYPE.itemsize + 4 * 6144))
    finally:
        st.close()


@pytest.mark.gpu
def test_device_image_equals_host_image_and_bad_images_are_refused():
    import torch
    spec = synthetic.ClipSpec(160, 96, 2, seed=64, rects=2, rect_size=(16, 40))
    frames = [np.ascontiguousarray(np.frombuffer(synthetic.packed(f), np.uint8)) for f in synthetic.generate(spec)]
    cfg = mav1cu.cli_config(spec.width, spec.height, q=125, turbo=1, tiles=0)
    jobs = mav1cu.plan(cfg, len(frames))
    st = mav1cu.Stream(cfg)
    try:
        sess = st.encode(jobs[0], torch.from_numpy(frames[jobs[0]["disp"]]).cuda().data_ptr(), True)
        cap = sess.export_capacity()
        host = _pinned(cap)
        dev = torch.zeros(cap, dtype=torch.uint8, device="cuda")
        sess.export(host.data_ptr(), cap, rec=True)
        sess.export(dev.data_ptr(), cap, rec=True)
        own = sess.export(rec=True)
        st.synchronize()
        h = host.numpy()
        n = int(h[:mav1cu.EXPORT_HEADER_DTYPE.itemsize].view(mav1cu.EXPORT_HEADER_DTYPE)[0]["bytes"])
        d = dev.cpu().numpy()
        o = np.ctypeslib.as_array(ctypes.cast(own, ctypes.POINTER(ctypes.c_uint8)), shape=(cap,))
        hdr = [x[:mav1cu.EXPORT_HEADER_DTYPE.itemsize].view(mav1cu.EXPORT_HEADER_DTYPE)[0] for x in (h, d, o)]
        assert [int(x["seq"]) for x in hdr] == [1, 2, 3]
        for a, b in zip(mav1cu.export_sections(h)[1:], mav1cu.export_sections(d)[1:]):
            assert np.array_equal(a, b)
        for a, b in zip(mav1cu.export_sections(h)[1:], mav1cu.export_sections(o)[1:]):
            assert np.array_equal(a, b)
        assert mav1cu.export_sections(h)[5] is not None
        assert n > 0
        # refused before any device work: too small, unaligned, pageable host memory
        lib = sess.lib
        assert lib.mav1cu_export(sess.h, host.data_ptr(), cap - 1, 0) == -1
    finally:
        st.close()
    st = mav1cu.Stream(cfg)
    try:
        sess = st.encode(jobs[0], torch.from_numpy(frames[jobs[0]["disp"]]).cuda().data_ptr(), True)
        cap = sess.export_capacity()
        host = _pinned(cap + 64)
        assert sess.lib.mav1cu_export(sess.h, host.data_ptr() + 4, cap, 0) == -1
    finally:
        st.close()
    st = mav1cu.Stream(cfg)
    try:
        sess = st.encode(jobs[0], torch.from_numpy(frames[jobs[0]["disp"]]).cuda().data_ptr(), True)
        cap = sess.export_capacity()
        pageable = np.zeros(cap + 64, np.uint8)
        addr = (pageable.ctypes.data + 15) & ~15
        assert sess.lib.mav1cu_export(sess.h, addr, cap, 0) == -1
        assert b"neither mapped" in sess.lib.mav1cu_error_string(sess.h)
    finally:
        st.close()
