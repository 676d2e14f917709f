"""ORACLE — test infrastructure only (imported by tests/, the smoke check and
bench.py's CPU-baseline leg; never by the product).

ctypes access to oracle/_ref/libmav1ref.so: the reference encoder's scalar
CPU path built from its own sources (see oracle/Makefile). Provides
  - encode(): the mav1.h queue API end to end (IVF packets, reconstructions,
    decision dump), exactly like the reference CLI tools/mav1enc.c;
  - a per-stage trace hook that snapshots the backend's inputs and outputs of
    every frame (run_frame_core's stages), for stage-level parity tests;
  - direct stage runners for the CPU baseline timing.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libmav1ref.so")
# the same driver built with the CUDA backend (backend_cuda.c) behind the vtable
HYB_PATH = os.path.join(HERE, "_ref", "libmav1hyb.so")

STAGE = dict(PARAMS=0, ME=1, ANALYZE=2, EDGE=3, RECON=4, FINFO=5, FILTER=6, CDEFSEL=7, LRSEL=8, RESTORE=9, DONE=10)
OBUF = dict(SRC=0, REC=1, REF=2, GOLD=3, PARAMS=4, MATS=5, MVFIELD=6, MVGOLD=7, BLOCKS=8, SBS=9, COEFS=10,
            LFMASK=11, CDEFBUF=12, DBK=13, LROUT=14, LRUNITS=15, ACOSTS=16, AINFOS=17, HPEL=18, CDEF_CHOICE=19)

CONFIG_FIELDS = ["width", "height", "qindex", "use_metal", "keyint", "tx_search", "tx_depth", "loop_filter", "cdef",
                 "restoration", "tile_cols_log2", "intra_edge_filter", "nonref_odd", "fast", "multi_ref", "altref",
                 "leaf", "switchable_interp", "lr_test", "me_range", "threads", "turbo"]


class Mav1Config(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in CONFIG_FIELDS]


HOOK = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p)

_libs = {}


def available(path=LIB_PATH):
    return os.path.exists(path)


def lib(path=LIB_PATH):
    if path not in _libs:
        if not available(path):
            raise RuntimeError(f"oracle not built ({path}); run make -C oracle")
        L = ctypes.CDLL(path)
        vp = ctypes.c_void_p
        L.mav1_default_config.argtypes = [ctypes.POINTER(Mav1Config), ctypes.c_int, ctypes.c_int]
        L.mav1_create.argtypes = [ctypes.POINTER(Mav1Config), ctypes.c_char_p, ctypes.c_size_t]
        L.mav1_create.restype = vp
        L.mav1_destroy.argtypes = [vp]
        L.mav1_send_frame.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_int)]
        L.mav1_receive_packet.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_size_t)]
        L.mav1_get_recon.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(ctypes.c_int)]
        L.oref_set_hook.argtypes = [HOOK, vp]
        L.oref_set_backend_factory.argtypes = [vp]
        L.oref_buf.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_size_t)]
        L.oref_buf.restype = vp
        L.oref_geometry.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
        L.oref_frame_state.argtypes = [vp, ctypes.POINTER(ctypes.c_int32)]
        L.oref_struct_sizes.argtypes = [ctypes.POINTER(ctypes.c_int32)]
        L.oref_run_stage.argtypes = [vp, ctypes.c_int]
        L.oref_set_num_cdef_presets.argtypes = [vp, ctypes.c_int]
        _libs[path] = L
    return _libs[path]


def cli_config(width, height, q=100, cpu=True, path=LIB_PATH, keyint=0, lf=1, cdef=1, txs=1, txd=1, lr=1, lr_test=0, sw=1,
               fast=0, turbo=0, golden=0, altref=0, leaf=0, edge=1, tiles=-1, me_range=32):
    """Mav1Config exactly as tools/mav1enc.c:36-104 builds it from its flags."""
    cfg = Mav1Config()
    lib(path).mav1_default_config(ctypes.byref(cfg), width, height)
    if turbo:
        fast = 1
    cfg.qindex = q
    cfg.use_metal = 0 if cpu else 1
    cfg.keyint = keyint
    cfg.loop_filter = lf
    cfg.cdef = cdef
    cfg.tx_search = txs
    cfg.tx_depth = txd
    cfg.restoration = lr
    cfg.lr_test = lr_test
    cfg.switchable_interp = sw
    cfg.me_range = me_range
    cfg.fast = fast
    cfg.turbo = turbo
    cfg.multi_ref = golden
    cfg.altref = altref
    cfg.leaf = leaf
    cfg.nonref_odd = 0
    cfg.intra_edge_filter = edge
    cfg.tile_cols_log2 = tiles if tiles >= 0 else (2 if turbo else 3 if fast else 0)
    if fast:
        cfg.tx_search = cfg.tx_depth = cfg.restoration = cfg.switchable_interp = 0
    return cfg


def buf(e, which):
    size = ctypes.c_size_t()
    p = lib().oref_buf(e, OBUF[which], ctypes.byref(size))
    return p, size.value


def snapshot(e, which, nbytes=None):
    p, size = buf(e, which)
    n = size if nbytes is None else min(nbytes, size)
    return np.frombuffer(ctypes.string_at(p, n), np.uint8).copy()


def geometry(e):
    g = (ctypes.c_int64 * 15)()
    lib().oref_geometry(e, g)
    keys = ["w", "h", "mi_cols", "mi_rows", "sb_cols", "sb_rows", "num_sbs", "tile_cols", "tile_w_sb", "frame_bytes",
            "num_cdef_presets", "stride0", "stride1", "offset1", "offset2"]
    return dict(zip(keys, list(g)))


def frame_state(e):
    s = (ctypes.c_int32 * 9)()
    lib().oref_frame_state(e, s)
    keys = ["frame_kind", "nonref", "leafopt", "order_hint", "is_key", "base_q_idx", "num_cdef_presets", "cdef_bits",
            "reference_select"]
    return dict(zip(keys, list(s)))


def struct_sizes():
    s = (ctypes.c_int32 * 8)()
    lib().oref_struct_sizes(s)
    return list(s)


class Trace:
    """Per-frame snapshots of the backend's inputs and outputs, captured by
    the stage hook of run_frame_core."""

    CAPTURE = {
        STAGE["PARAMS"]: ["PARAMS", "SRC", "REF", "GOLD", "REC", "COEFS", "MVFIELD", "MVGOLD"],
        STAGE["ME"]: ["MVFIELD", "MVGOLD"],
        STAGE["ANALYZE"]: ["BLOCKS", "SBS", "ACOSTS", "AINFOS"],
        STAGE["EDGE"]: ["BLOCKS"],
        STAGE["RECON"]: ["REC", "BLOCKS", "COEFS"],
        STAGE["FINFO"]: ["LFMASK"],
        STAGE["FILTER"]: ["REC", "CDEFBUF"],
        STAGE["CDEFSEL"]: ["REC", "CDEF_CHOICE"],
        STAGE["LRSEL"]: ["PARAMS", "LRUNITS", "DBK"],
        STAGE["RESTORE"]: ["LROUT"],
        STAGE["DONE"]: ["REC"],
    }

    def __init__(self, stages=None):
        self.frames = []
        self.stages = stages
        self.geom = None

        def hook(user, stage, e):
            if self.stages is not None and stage not in self.stages:
                return
            if stage == STAGE["PARAMS"]:
                self.frames.append({"state": frame_state(e)})
                if self.geom is None:
                    self.geom = geometry(e)
                    self.mats = snapshot(e, "MATS")
            fr = self.frames[-1]
            if stage == STAGE["FILTER"]:
                fr["npresets_filter"] = frame_state(e)["num_cdef_presets"]
            for name in self.CAPTURE.get(stage, []):
                fr[(stage, name)] = snapshot(e, name)

        self.cb = HOOK(hook)


def _planes(frame, w, h):
    cw, ch = (w + 1) // 2, (h + 1) // 2
    arrs = [np.ascontiguousarray(frame[0], np.uint8), np.ascontiguousarray(frame[1], np.uint8),
            np.ascontiguousarray(frame[2], np.uint8)]
    ptrs = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in arrs])
    strides = (ctypes.c_int * 3)(w, cw, cw)
    return arrs, ptrs, strides


def encode(frames, cfg, trace=None, factory=None, path=LIB_PATH):
    """Encodes the frames through mav1_send_frame / mav1_receive_packet like
    tools/mav1enc.c. Returns (packets, recons): the temporal units and the
    shown reconstruction of each (I420 planes). With path=HYB_PATH and
    cuda=True in cfg.use_metal the CUDA backend codes every frame."""
    L = lib(path)
    if factory == "cuda":
        factory = ctypes.cast(L.backend_cuda_create, ctypes.c_void_p)
    L.oref_set_hook(trace.cb if trace else HOOK(), None)
    L.oref_set_backend_factory(factory)
    err = ctypes.create_string_buffer(256)
    e = L.mav1_create(ctypes.byref(cfg), err, 256)
    if not e:
        L.oref_set_hook(HOOK(), None)
        raise RuntimeError("mav1_create: " + err.value.decode())
    w, h = cfg.width, cfg.height
    cw, ch = (w + 1) // 2, (h + 1) // 2
    packets, recons = [], []

    def drain():
        pkt = ctypes.c_void_p()
        n = ctypes.c_size_t()
        while L.mav1_receive_packet(e, ctypes.byref(pkt), ctypes.byref(n)) == 0:
            packets.append(ctypes.string_at(pkt, n.value))
            ctypes.CDLL(None).free(pkt)
            rec = [np.zeros((h, w), np.uint8), np.zeros((ch, cw), np.uint8), np.zeros((ch, cw), np.uint8)]
            ptrs = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in rec])
            strides = (ctypes.c_int * 3)(w, cw, cw)
            L.mav1_get_recon(e, ptrs, strides)
            recons.append(rec)

    try:
        for fr in frames:
            arrs, ptrs, strides = _planes(fr, w, h)
            if L.mav1_send_frame(e, ptrs, strides):
                raise RuntimeError("mav1_send_frame failed")
            drain()
        L.mav1_send_frame(e, None, None)
        drain()
    finally:
        L.mav1_destroy(e)
        L.oref_set_hook(HOOK(), None)
        L.oref_set_backend_factory(None)
    return packets, recons


def ivf_bytes(packets, w, h, fps=(30, 1)):
    """IVF container exactly as tools/mav1enc.c writes it."""
    import struct
    out = bytearray(b"DKIF" + struct.pack("<HH4sHHIIII", 0, 32, b"AV01", w, h, fps[0], fps[1], len(packets), 0))
    for i, p in enumerate(packets):
        out += struct.pack("<IQ", len(p), i) + p
    return bytes(out)
