"""Stage-level parity harness: replays the oracle's per-frame backend inputs
through the CUDA stages (via the C ABI) and compares every output with the
oracle's, field by field. Each stage gets the oracle's own inputs, so a
mismatch is attributed to exactly one stage."""
import numpy as np

import mav1cu
import oracle
import synthetic
from mav1cu import BLOCK_DTYPE, LRUNIT_DTYPE, PARAMS_DTYPE, SB_DTYPE

ST = oracle.STAGE
NUM_NODES, A_SLOTS = 85, 13


def trace_clip(spec, nframes, **flags):
    frames = list(synthetic.generate(spec, nframes))
    cfg = oracle.cli_config(spec.width, spec.height, **flags)
    tr = oracle.Trace()
    packets, recons = oracle.encode(frames, cfg, trace=tr)
    return tr, cfg, frames, packets, recons


def params_of(fr):
    return fr[(ST["PARAMS"], "PARAMS")][:392].copy()


def level_slots(p, level):
    turbo_square = (p["turbo"] & 1) and (not p["frame_is_intra"] or (p["turbo"] & 256))
    if level == 3 or turbo_square:
        return 1
    if level == 2 or p["fast"]:
        return 5
    return A_SLOTS


def node_base(level):
    return (0, 1, 5, 21)[level]


class FrameCheck:
    """Runs the CUDA stages of one traced frame against the oracle's snapshots."""

    def __init__(self, sess, tr, cfg, fr):
        self.s, self.tr, self.cfg, self.fr = sess, tr, cfg, fr
        self.g = tr.geom
        self.fb = self.g["frame_bytes"]
        self.nsb = self.g["num_sbs"]
        self.params = params_of(fr)
        self.p = self.params.view(PARAMS_DTYPE)[0]
        self.state = fr["state"]

    def snap(self, stage, name, nbytes=None):
        a = self.fr[(ST[stage], name)]
        return a if nbytes is None else a[:nbytes]

    def frame_inputs(self):
        s, fb = self.s, self.fb
        s.set_params(self.params)
        s.upload("SRC", self.snap("PARAMS", "SRC", fb))
        s.upload("REF", self.snap("PARAMS", "REF", fb))
        s.upload("GOLD", self.snap("PARAMS", "GOLD", fb))
        s.upload("MATS", self.tr.mats[:15 * 4096 * 4])

    # ---- per-stage checks: each returns {output: mismatch count} -------------
    def me(self):
        if self.p["frame_is_intra"]:
            return {}
        self.frame_inputs()
        self.s.motion_search()
        n = self.nsb * NUM_NODES * 2 * 4
        out = {"mvfield": diff(self.s.download("MVFIELD", count=n), self.snap("ME", "MVFIELD", n))}
        if self.p["golden"]:
            out["mvgold"] = diff(self.s.download("MVGOLD", count=n), self.snap("ME", "MVGOLD", n))
        return out

    def analyze(self):
        self.frame_inputs()
        n = self.nsb * NUM_NODES * 2 * 4
        self.s.upload("MVFIELD", self.snap("ME", "MVFIELD", n))
        self.s.upload("MVGOLD", self.snap("ME", "MVGOLD", n))
        self.s.analyze()
        out = {}
        costs = self.s.download("ACOSTS", np.int64)
        infos = self.s.download("AINFOS", count=self.s.size("AINFOS")).view(BLOCK_DTYPE)
        rc = self.snap("ANALYZE", "ACOSTS", self.s.size("ACOSTS")).view(np.int64)
        ri = self.snap("ANALYZE", "AINFOS", self.s.size("AINFOS")).view(BLOCK_DTYPE)
        idx = []
        for level in range(4):
            ns = level_slots(self.p, level)
            for sb in range(self.nsb):
                for i in range(1 << (2 * level)):
                    base = sb * NUM_NODES * A_SLOTS + (node_base(level) + i) * A_SLOTS
                    idx.extend(range(base, base + ns))
        idx = np.array(idx)
        out["acosts"] = int((costs[idx] != rc[idx]).sum())
        live = idx[rc[idx] >= 0]
        out["ainfos"] = blocks_diff(infos[live], ri[live], skip=("eob", "coef_off"))
        out.update(self.blocks_sbs("ANALYZE"))
        return out

    def blocks_sbs(self, stage, sbs_ref_stage="ANALYZE"):
        blocks = self.s.download("BLOCKS", count=self.s.size("BLOCKS")).view(BLOCK_DTYPE)
        sbs = self.s.download("SBS", count=self.s.size("SBS")).view(SB_DTYPE)
        rb = self.snap(stage, "BLOCKS", self.s.size("BLOCKS")).view(BLOCK_DTYPE)
        rs = self.snap("ANALYZE", "SBS", self.s.size("SBS")).view(SB_DTYPE)
        out = {"sbs": int((sbs != rs).sum())}
        sel = np.concatenate([np.arange(r["first_block"], r["first_block"] + r["num_blocks"]) for r in rs])
        out["blocks"] = blocks_diff(blocks[sel], rb[sel])
        return out

    def upload_blocks(self, stage):
        self.s.upload("BLOCKS", self.snap(stage, "BLOCKS", self.s.size("BLOCKS")))
        self.s.upload("SBS", self.snap("ANALYZE", "SBS", self.s.size("SBS")))

    def edge(self):
        if not self.cfg.intra_edge_filter:
            return {}
        self.frame_inputs()
        self.upload_blocks("ANALYZE")
        self.s.edge_types()
        return {"blocks": self.blocks_sbs("EDGE")["blocks"]}

    def recon(self):
        self.frame_inputs()
        self.upload_blocks("EDGE")
        self.s.upload("REC", self.snap("PARAMS", "REC", self.fb))
        self.s.upload("COEFS", self.snap("PARAMS", "COEFS", self.s.size("COEFS")))
        self.s.recon()
        out = {"rec": diff(self.s.download("REC", count=self.fb), self.snap("RECON", "REC", self.fb))}
        out["coefs"] = diff(self.s.download("COEFS", np.int32), self.snap("RECON", "COEFS", self.s.size("COEFS")).view(np.int32))
        out["blocks"] = self.blocks_sbs("RECON")["blocks"]
        return out

    def filtered(self):
        lf_on = any(self.p["lf_level"])
        cdef_off = (self.state["leafopt"] & 4) != 0
        return lf_on or (self.state["num_cdef_presets"] and not cdef_off) or not self.cfg.turbo

    def finfo(self):
        if not self.filtered():
            return {}
        self.frame_inputs()
        self.upload_blocks("RECON")
        self.s.filter_info()
        n = self.g["mi_rows"] * self.g["mi_cols"]
        return {"lfmask": diff(self.s.download("LFMASK", count=n), self.snap("FINFO", "LFMASK", n))}

    def filter(self):
        if not self.filtered():
            return {}
        self.frame_inputs()
        n = self.g["mi_rows"] * self.g["mi_cols"]
        self.s.upload("LFMASK", self.snap("FINFO", "LFMASK", n))
        self.s.upload("REC", self.snap("RECON", "REC", self.fb))
        np_ = self.fr["npresets_filter"]
        self.s.filter(np_)
        out = {"rec": diff(self.s.download("REC", count=self.fb), self.snap("FILTER", "REC", self.fb))}
        if np_:
            k = np_ * self.fb
            out["cdefbuf"] = diff(self.s.download("CDEFBUF", count=k), self.snap("FILTER", "CDEFBUF", k))
        return out

    def cdef_select(self):
        cdef_off = (self.state["leafopt"] & 4) != 0
        if not (self.cfg.cdef and self.cfg.qindex > 0 and not cdef_off):
            return {}
        self.frame_inputs()
        self.s.upload("REC", self.snap("FILTER", "REC", self.fb))
        np_ = self.state["num_cdef_presets"]
        self.s.upload("CDEFBUF", self.snap("FILTER", "CDEFBUF", np_ * self.fb))
        self.s.cdef_select(np_)
        return {
            "rec": diff(self.s.download("REC", count=self.fb), self.snap("CDEFSEL", "REC", self.fb)),
            "cdef_choice": diff(self.s.download("CDEF_CHOICE", count=self.nsb), self.snap("CDEFSEL", "CDEF_CHOICE", self.nsb)),
        }

    def restore(self):
        if (ST["RESTORE"], "LROUT") not in self.fr:
            return {}
        self.frame_inputs()
        self.s.set_params(self.fr[(ST["LRSEL"], "PARAMS")][:392].copy())
        self.s.upload("REC", self.snap("CDEFSEL", "REC", self.fb))
        self.s.upload("DBK", self.snap("LRSEL", "DBK", self.fb))
        self.s.upload("LROUT", self.snap("CDEFSEL", "REC", self.fb))
        self.s.upload("LRUNITS", self.snap("LRSEL", "LRUNITS", self.s.size("LRUNITS")))
        self.s.restore()
        return {"lrout": diff(self.s.download("LROUT", count=self.fb), self.snap("RESTORE", "LROUT", self.fb))}

    def lr_search(self):
        """The loop-restoration search (lr_select, lr_search.c:244-359) on the
        oracle's CDEF output and deblocked frame: every unit record in use and
        each plane's lr_type."""
        if (ST["LRSEL"], "LRUNITS") not in self.fr:
            return {}
        self.frame_inputs()
        self.s.upload("REC", self.snap("CDEFSEL", "REC", self.fb))
        self.s.upload("DBK", self.snap("LRSEL", "DBK", self.fb))
        self.s.lr_search(int(self.cfg.lr_test))
        p = self.p
        n = int(p["lr_unit_off"][2] + p["lr_unit_rows"][2] * p["lr_unit_cols"][2])
        got = self.s.download("LRUNITS", LRUNIT_DTYPE, count=n)
        want = self.snap("LRSEL", "LRUNITS", n * LRUNIT_DTYPE.itemsize).view(LRUNIT_DTYPE)
        gp = self.s.download("PARAMS", np.uint8, count=392).view(PARAMS_DTYPE)[0]
        wp = self.fr[(ST["LRSEL"], "PARAMS")][:392].copy().view(PARAMS_DTYPE)[0]
        bad = [i for i in range(n) if got[i].tobytes() != want[i].tobytes()]
        return {"lrunits": len(bad), "lr_type": int((gp["lr_type"] != wp["lr_type"]).sum())}

    def chain(self):
        """Every stage on the device from the frame inputs only, in
        run_frame_core's order (encoder.c:599-657), the loop-restoration
        search included."""
        self.frame_inputs()
        self.s.upload("REC", self.snap("PARAMS", "REC", self.fb))
        self.s.upload("COEFS", self.snap("PARAMS", "COEFS", self.s.size("COEFS")))
        self.s.frame_core()
        if self.filtered():
            self.s.filter_info()
            self.s.filter(self.fr["npresets_filter"])
        use_lr = (ST["RESTORE"], "LROUT") in self.fr
        if use_lr:
            self.s.copy("DBK", "REC")
        cdef_off = (self.state["leafopt"] & 4) != 0
        if self.cfg.cdef and self.cfg.qindex > 0 and not cdef_off:
            self.s.cdef_select(self.state["num_cdef_presets"])
        final = "REC"
        if use_lr:
            self.s.lr_search(int(self.cfg.lr_test))
            self.s.copy("LROUT", "REC")
            self.s.restore()
            final = "LROUT"
        out = {"rec": diff(self.s.download(final, count=self.fb), self.snap("DONE", "REC", self.fb))}
        out["coefs"] = diff(self.s.download("COEFS", np.int32), self.snap("RECON", "COEFS", self.s.size("COEFS")).view(np.int32))
        out.update(self.blocks_sbs("RECON"))
        return out


def diff(a, b):
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()[: a.size]
    return int((a != b).sum())


def blocks_diff(a, b, skip=()):
    n = 0
    for name in BLOCK_DTYPE.names:
        if name in skip:
            continue
        n += int((a[name] != b[name]).sum())
    return n


def first_block_mismatch(a, b, skip=()):
    for i in range(len(a)):
        for name in BLOCK_DTYPE.names:
            if name in skip:
                continue
            if np.any(a[i][name] != b[i][name]):
                return i, name, a[i], b[i]
    return None


STAGES = ("me", "analyze", "edge", "recon", "finfo", "filter", "cdef_select", "lr_search", "restore", "chain")


def check_all(sess, tr, cfg, stages=STAGES):
    """[(frame index, state, {stage: {output: mismatches}})]"""
    res = []
    for k, fr in enumerate(tr.frames):
        fc = FrameCheck(sess, tr, cfg, fr)
        res.append((k, fr["state"], {st: getattr(fc, st)() for st in stages}))
    return res


# ---- whole-stream comparisons -------------------------------------------------------
import os
import re

_TABLES = None


def spec_tables():
    """The normative tables the library is compiled with (csrc/spec_tables_gen.h)."""
    global _TABLES
    if _TABLES is None:
        path = os.path.join(os.path.dirname(mav1cu.__file__), "csrc", "spec_tables_gen.h")
        text = open(path).read()
        _TABLES = {}
        for name, dims, body in re.findall(r"#define MAV1T_(\w+)_DIMS ((?:\[\d+\])+)\n#define MAV1T_\1 \{(.*?)\}", text, re.S):
            shape = [int(d) for d in re.findall(r"\d+", dims)]
            vals = [int(v) for v in re.findall(r"-?\d+", body.replace("\\", " "))]
            _TABLES[name] = np.array(vals, np.int64).reshape(shape)
    return _TABLES


def tx_layout(b, plane, p):
    """(txSz, [(startX, startY)]) of the transform blocks code_plane codes for
    plane `plane` of block b (k_recon.h:190-291)."""
    T = spec_tables()
    bs = int(b["bsize"])
    sub = 1 if plane else 0
    if p["lossless"]:
        tx = 0
    elif plane:
        uv = int(T["Max_Tx_Size_Rect"][T["Subsampled_Size"][bs][1][1]])
        tw, th = T["Tx_Width"][uv], T["Tx_Height"][uv]
        tx = uv
        if tw == 64 or th == 64:
            tx = 9 if tw == 16 else 10 if th == 16 else 3
    else:
        tx = int(T["Max_Tx_Size_Rect"][bs])
        for _ in range(int(b["tx_depth"]) if not b["is_inter"] else 0):
            tx = int(T["Split_Tx_Size"][tx])
    psz = int(T["Subsampled_Size"][bs][sub][sub])
    n4w, n4h = int(T["Num_4x4_Blocks_Wide"][psz]), int(T["Num_4x4_Blocks_High"][psz])
    bx, by = (int(b["mi_col"]) >> sub) * 4, (int(b["mi_row"]) >> sub) * 4
    sx, sy = int(T["Tx_Width"][tx]) >> 2, int(T["Tx_Height"][tx]) >> 2
    starts = []
    for y in range(0, n4h, sy):
        for x in range(0, n4w, sx):
            X, Y = bx + 4 * x, by + 4 * y
            if X >= (p["mi_cols"] * 4) >> sub or Y >= (p["mi_rows"] * 4) >> sub:
                continue
            starts.append((X, Y))
    return tx, starts


def used_coefs(blocks, sbs, p):
    """Indices of the coefficient buffer the frame's blocks write."""
    T = spec_tables()
    idx = []
    for r in sbs:
        for b in blocks[r["first_block"]: r["first_block"] + r["num_blocks"]]:
            for plane in range(3):
                tx, starts = tx_layout(b, plane, p)
                w, h = int(T["Tx_Width"][tx]), int(T["Tx_Height"][tx])
                n = min(32, w) * min(32, h)
                for k in range(len(starts)):
                    o = int(b["coef_off"][plane]) + k * w * h
                    idx.append(np.arange(o, o + n))
    return np.concatenate(idx) if idx else np.zeros(0, np.int64)


def visible(frame, g):
    """The frame's displayed samples (w x h luma, (w+1)/2 x (h+1)/2 chroma) from a padded buffer."""
    w, h = g["w"], g["h"]
    s0, s1 = g["stride"][0], g["stride"][1]
    o1, o2 = g["offset"][1], g["offset"][2]
    cw, ch = (w + 1) // 2, (h + 1) // 2
    y = frame[: s0 * g["plane_h"][0]].reshape(-1, s0)[:h, :w]
    u = frame[o1: o1 + s1 * g["plane_h"][1]].reshape(-1, s1)[:ch, :cw]
    v = frame[o2: o2 + s1 * g["plane_h"][2]].reshape(-1, s1)[:ch, :cw]
    return np.concatenate([y.ravel(), u.ravel(), v.ravel()])


def stream_vs_oracle(tr, frames, flags, spec):
    """Codes the traced clip through the device stream (mav1cu_stream, both
    engines) and compares every frame's writer inputs and reconstruction with
    the oracle's, in coding order. Returns [(frame, {output: mismatches})]."""
    cfg = mav1cu.cli_config(spec.width, spec.height, **flags)
    jobs = mav1cu.plan(cfg, len(frames))
    assert len(jobs) == len(tr.frames)
    st = mav1cu.Stream(cfg)
    g = mav1cu.geometry(spec.width, spec.height)
    dev = [np.ascontiguousarray(np.frombuffer(synthetic.packed(f), np.uint8)) for f in frames]
    import torch
    dframes = [torch.from_numpy(d).cuda() for d in dev]
    res = []
    try:
        for k, (job, fr) in enumerate(zip(jobs, tr.frames)):
            sess = st.encode(job, dframes[job["disp"]].data_ptr(), True)
            st.synchronize()
            p = params_of(fr).view(PARAMS_DTYPE)[0]
            fb = g["frame_bytes"]
            out = {}
            rec = sess.download("REC", count=fb)
            done = fr[(ST["DONE"], "REC")][:fb]
            out["rec"] = int((visible(rec, g) != visible(done, g)).sum())
            blocks = sess.download("BLOCKS", count=sess.size("BLOCKS")).view(BLOCK_DTYPE)
            sbs = sess.download("SBS", count=sess.size("SBS")).view(SB_DTYPE)
            rb = fr[(ST["RECON"], "BLOCKS")][: sess.size("BLOCKS")].view(BLOCK_DTYPE)
            rs = fr[(ST["ANALYZE"], "SBS")][: sess.size("SBS")].view(SB_DTYPE)
            out["sbs"] = int((sbs != rs).sum())
            sel = np.concatenate([np.arange(r["first_block"], r["first_block"] + r["num_blocks"]) for r in rs])
            out["blocks"] = blocks_diff(blocks[sel], rb[sel])
            coefs = sess.download("COEFS", np.int32)
            rcoefs = fr[(ST["RECON"], "COEFS")][: sess.size("COEFS")].view(np.int32)
            used = used_coefs(rb, rs, p)
            out["coefs"] = int((coefs[used] != rcoefs[used]).sum())
            if (ST["CDEFSEL"], "CDEF_CHOICE") in fr and fr["state"]["leafopt"] & 4 == 0:
                n = g["num_sbs"]
                out["cdef_choice"] = int((sess.download("CDEF_CHOICE", count=n) != fr[(ST["CDEFSEL"], "CDEF_CHOICE")][:n]).sum())
            res.append((k, out))
    finally:
        st.close()
    return res


# ---- compact export of the writer inputs ------------------------------------------


def pack_writer_inputs(blocks, sbs, coefs, cdef, p):
    """The compact export image's sections (mav1cu_export) restated from the
    dense BLOCKS / SBS / COEFS / CDEF_CHOICE buffers: the blocks in use with
    first_block and coef_off rewritten, and a level run that opens with
    zeros as long as the largest zero plane of a coded block, followed by
    the levels of every coded plane (eob != 0) of every coded block over the
    transform blocks the writer visits (tile_writer.c:437-456), up to the
    last level it may read."""
    T = spec_tables()

    def region(b, plane):
        # transform blocks tw * th apart; the writer reads the last one only
        # inside its adjusted (at most 32 x 32) transform
        tx, starts = tx_layout(b, plane, p)
        w, h = int(T["Tx_Width"][tx]), int(T["Tx_Height"][tx])
        return (len(starts) - 1) * w * h + min(32, w) * min(32, h) if starts else 0

    used = [blocks[r["first_block"]: r["first_block"] + r["num_blocks"]] for r in sbs]
    zrun = 0
    for bl in used:
        for b in bl:
            if b["eob"].any():
                zrun = max([zrun] + [region(b, pl) for pl in range(3) if not b["eob"][pl]])
    out_sbs = sbs.copy()
    out_blocks = np.concatenate(used).copy() if used else np.zeros(0, BLOCK_DTYPE)
    levels = [np.zeros(zrun, np.int32)]
    pos, k = zrun, 0
    for i, bl in enumerate(used):
        out_sbs[i]["first_block"] = k
        for b in bl:
            nb = out_blocks[k]
            for pl in range(3):
                if b["eob"].any() and b["eob"][pl]:
                    n = region(b, pl)
                    o = int(b["coef_off"][pl])
                    levels.append(np.asarray(coefs[o: o + n], np.int32))
                    nb["coef_off"][pl] = pos
                    pos += n
                else:
                    nb["coef_off"][pl] = 0
            k += 1
    return dict(sbs=out_sbs, cdef=np.asarray(cdef[: len(sbs)], np.int8), blocks=out_blocks,
                levels=np.concatenate(levels), zero_run=zrun)


def export_vs_packed(image, blocks, sbs, coefs, cdef, p):
    """Mismatch counts between an export image (uint8 array) and the packing
    of the dense buffers it was made from."""
    h, isbs, icdef, iblocks, ilevels, irec = mav1cu.export_sections(image)
    want = pack_writer_inputs(blocks, sbs, coefs, cdef, p)
    out = dict(zero_run=int(h["zero_run"] != want["zero_run"]),
               num_blocks=int(h["num_blocks"] != len(want["blocks"])),
               num_coefs=int(h["num_coefs"] != len(want["levels"])))
    out["sbs"] = int((isbs != want["sbs"]).sum()) if len(isbs) == len(want["sbs"]) else -1
    out["cdef"] = int((icdef != want["cdef"]).sum())
    out["blocks"] = int((iblocks != want["blocks"]).sum()) if len(iblocks) == len(want["blocks"]) else -1
    out["levels"] = int((ilevels != want["levels"]).sum()) if len(ilevels) == len(want["levels"]) else -1
    nbytes = (mav1cu.EXPORT_HEADER_DTYPE.itemsize + len(isbs) * SB_DTYPE.itemsize + len(icdef) +
              len(iblocks) * BLOCK_DTYPE.itemsize + 4 * len(ilevels) + mav1cu.PARAMS_DTYPE.itemsize +
              mav1cu.LRUNIT_DTYPE.itemsize * int(h["lr_units"]) + (0 if irec is None else len(irec)))
    out["bytes"] = int(h["bytes"] != nbytes)
    return out
