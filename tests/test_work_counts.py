"""The counting build's work counters (include/mav1cu_count.h) against the
same units derived on the CPU from the reference's own decisions.

The structural counts are restated from the reference's loops: the motion
search's full-pel candidates per node and stage (src/kernels/k_me.h:141-223:
me_node, me_refine_stage, me_cost with its decimated and row-subsampled
SADs), and the reconstruction's transform blocks, forward-transform passes,
quantised coefficients and predictions per block (src/kernels/k_recon.h:60-173
code_tx_block, :190-291 code_plane, :293-394 recon_block), evaluated over the
oracle's block decisions. On the GPU the counting library codes the same
frames and its counters must equal them exactly: the kernels do the
algorithmic work the reference defines, once."""
import numpy as np
import pytest

import mav1cu
import oracle
import parity
import synthetic
from mav1cu import BLOCK_DTYPE, SB_DTYPE

ST = oracle.STAGE
T_ME = dict(CR1=2, L3COPY=4, DEC=32, CR2=64, REF2=512, LEAF_NO8=1024, L3SUB=4096, G3COPY=16384, RSUB=65536,
            HME3=131072)
TX_16X32, TX_32X16, TX_32X32 = 9, 10, 3


def me_fullpel_pairs(p):
    """(full-resolution, decimated) SAD byte pairs of one frame's motion
    search: every valid, non-copied node of every level of every superblock,
    per reference searched (k_me.h:141-223)."""
    if p["frame_is_intra"]:
        return 0, 0
    tb = int(p["turbo"])
    on = lambda f: bool(tb & T_ME[f])
    leaf = bool(p["leaf"]) and not p["frame_is_intra"]
    full = dec = 0
    for ref in range(2 if p["golden"] else 1):
        for sb in range(int(p["sb_rows"]) * int(p["sb_cols"])):
            sbr, sbc = divmod(sb, int(p["sb_cols"]))
            for level in range(4):
                n, w = 1 << level, 64 >> level
                for i in range(n * n):
                    x, y = sbc * 64 + (i % n) * w, sbr * 64 + (i // n) * w
                    if x >= p["frame_w"] or y >= p["frame_h"]:
                        continue
                    copy = level == 3 and (on("L3COPY") or (on("LEAF_NO8") and leaf))
                    if ref == 1 and level == 3 and on("G3COPY") and leaf:
                        copy = True
                    if copy:
                        continue
                    rng = int(p["me_range"])
                    step, stages = 1, 1
                    if level > 0:
                        rng = min(rng, 1 if on("CR1") else 2 if on("CR2") else 4)
                    else:
                        step = 8 if on("HME3") else 4
                        rng = (rng // step) * step
                        stages = 3 if on("HME3") else 2
                    if level == 3 and on("L3SUB"):
                        stages = 0
                    for stage in range(stages):
                        if stage > 0:
                            if stage == 1 and on("HME3"):
                                rng, step = 4, 4
                            else:
                                rng, step = (2 if on("REF2") else 3), 1
                        side = 2 * (rng // step) + 1
                        count = 1 + side * side
                        if on("DEC") and step >= 4:
                            dec += count * (w // 4) ** 2
                        else:
                            rs = 2 if on("RSUB") and step == 1 else 1
                            full += count * (w // rs) * w
    return full, dec


def recon_units(p, blocks, sbs):
    """Forward-transform multiply-accumulates, quantised coefficients and
    intra / inter predicted samples of one frame's reconstruction."""
    T = parity.spec_tables()
    bw = lambda bs: 4 * int(T["Num_4x4_Blocks_Wide"][bs])
    bh = lambda bs: 4 * int(T["Num_4x4_Blocks_High"][bs])

    def uv_tx(bs):
        t = int(T["Max_Tx_Size_Rect"][int(T["Subsampled_Size"][bs][1][1])])
        if T["Tx_Width"][t] == 64 or T["Tx_Height"][t] == 64:
            return TX_16X32 if T["Tx_Width"][t] == 16 else TX_32X16 if T["Tx_Height"][t] == 16 else TX_32X32
        return t

    out = dict(fwd_mac=0, quant=0, rec_intra_px=0, rec_inter_px=0)
    assert not p["lossless"] and not p["tx_search"] and not p["tx_mode_select"]
    for sb in range(int(p["sb_rows"]) * int(p["sb_cols"])):
        s = sbs[sb]
        for k in range(min(int(s["num_blocks"]), 64)):
            b = blocks[int(s["first_block"]) + k]
            bs, inter = int(b["bsize"]), bool(b["is_inter"])
            if inter:
                comp = int(b["ref_frame1"]) > 0
                if p["switchable_interp"] and not comp:
                    out["rec_inter_px"] += 9 * bw(bs) * bh(bs)  # the dual-filter search (k_recon.h:304-328)
                for pl in range(3):
                    sub = pl > 0
                    out["rec_inter_px"] += (2 if comp else 1) * (bw(bs) >> sub) * (bh(bs) >> sub)
            for pl in range(3):
                sub = int(pl > 0)
                tx = int(T["Max_Tx_Size_Rect"][bs]) if pl == 0 else uv_tx(bs)
                psz = int(T["Subsampled_Size"][bs][sub][sub])
                n4w, n4h = int(T["Num_4x4_Blocks_Wide"][psz]), int(T["Num_4x4_Blocks_High"][psz])
                tw, th = int(T["Tx_Width"][tx]), int(T["Tx_Height"][tx])
                x0, y0 = (int(b["mi_col"]) >> sub) * 4, (int(b["mi_row"]) >> sub) * 4
                for y in range(0, n4h, th >> 2):
                    for x in range(0, n4w, tw >> 2):
                        if x0 + 4 * x >= (int(p["mi_cols"]) * 4) >> sub or y0 + 4 * y >= (int(p["mi_rows"]) * 4) >> sub:
                            continue
                        ktw, kth = min(32, tw), min(32, th)
                        out["fwd_mac"] += th * ktw * tw + kth * ktw * th
                        out["quant"] += kth * ktw
                        if not inter:
                            out["rec_intra_px"] += tw * th
    return out


CASE = (synthetic.CONFIGS["c0_352x288"], 5, dict(q=125, turbo=1, keyint=30, tiles=0))


def expected(trace):
    """Per frame in coding order: the derived counts."""
    res = []
    for fr in trace.frames:
        p = parity.params_of(fr).view(mav1cu.PARAMS_DTYPE)[0]
        nsb = int(p["sb_rows"]) * int(p["sb_cols"])
        blocks = fr[(ST["RECON"], "BLOCKS")][: nsb * 64 * BLOCK_DTYPE.itemsize].view(BLOCK_DTYPE)
        sbs = fr[(ST["ANALYZE"], "SBS")][: nsb * SB_DTYPE.itemsize].view(SB_DTYPE)
        full, dec = me_fullpel_pairs(p)
        res.append(dict(me_sad=full, me_dec_sad=dec, **recon_units(p, blocks, sbs)))
    return res


@pytest.mark.skipif(not oracle.available(), reason="oracle not built")
def test_derived_counts_are_structural():
    """CPU: the restated counts on the reference's decisions are positive
    where the frame has the work and zero where it has none (a key frame has
    no motion search, a leaf frame no intra blocks)."""
    spec, n, flags = CASE
    tr, cfg, frames, packets, recons = parity.trace_clip(spec, n, **flags)
    exp = expected(tr)
    kinds = [int(parity.params_of(fr).view(mav1cu.PARAMS_DTYPE)[0]["frame_is_intra"]) for fr in tr.frames]
    assert kinds[0] == 1 and exp[0]["me_sad"] == exp[0]["me_dec_sad"] == 0 and exp[0]["rec_intra_px"] > 0
    assert all(e["me_sad"] + e["me_dec_sad"] > 0 for e, k in zip(exp, kinds) if not k)
    assert all(e["fwd_mac"] > 0 and e["quant"] > 0 for e in exp)


@pytest.mark.gpu
@pytest.mark.skipif(not oracle.available(), reason="oracle not built")
def test_counting_build_matches_reference_structure():
    import torch

    spec, n, flags = CASE
    tr, cfg, frames, packets, recons = parity.trace_clip(spec, n, **flags)
    exp = expected(tr)
    lib_ = mav1cu.load_count_library()
    saved = mav1cu._lib
    mav1cu._lib = lib_
    try:
        ccfg = mav1cu.cli_config(spec.width, spec.height, **flags)
        jobs = mav1cu.plan(ccfg, n)
        dev = torch.from_numpy(np.stack([np.frombuffer(synthetic.packed(f), np.uint8) for f in frames])).cuda()
        st = mav1cu.Stream(ccfg)
        got = []
        try:
            for j in jobs:
                st.synchronize()
                lib_.mav1cu_work_reset()
                st.encode(j, dev[j["disp"]].data_ptr(), True)
                st.synchronize()
                got.append(mav1cu.work_read(lib_))
        finally:
            st.close()
    finally:
        mav1cu._lib = saved
    assert len(got) == len(exp)
    for i, (g, e) in enumerate(zip(got, exp)):
        for k, v in e.items():
            assert g[k] == v, (i, k, g[k], v)
        assert g["me_satd"] > 0 or e["me_sad"] + e["me_dec_sad"] == 0


def test_counting_library_exports():
    """The counting build loads without a GPU and exports the entry points of
    both headers."""
    import os
    import re
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    names = set()
    for h in ("mav1cu.h", "mav1cu_count.h"):
        text = re.sub(r"/\*.*?\*/", "", open(os.path.join(root, "include", h)).read(), flags=re.S)
        names |= set(re.findall(r"\b(mav1cu_\w+)\s*\(", text))
    lib_ = mav1cu.load_count_library()
    assert {"mav1cu_work_read", "mav1cu_work_reset", "mav1cu_work_int_peak"} <= names
    assert [n for n in sorted(names) if not hasattr(lib_, n)] == []
    assert len(mav1cu.WORK_NAMES) == 16
