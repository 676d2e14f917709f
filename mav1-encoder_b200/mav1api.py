"""Python binding of libmav1.so: the mav1 encoder API (the reference's
src/mav1.h, unchanged) on the B200 encode backend.

Encoder mirrors the queue API a caller of the reference uses (mav1_create,
mav1_send_frame, mav1_receive_packet, mav1_get_recon, mav1_destroy;
tools/mav1enc.c is such a caller); encode() runs a clip through it like the
reference CLI and returns the temporal units and the shown reconstructions;
ivf_bytes() wraps temporal units in the CLI's IVF container.

The library needs libmav1cu.so and a CUDA device; there is no CPU backend
(a configuration with use_metal = 0 is refused by mav1_create).
"""
import ctypes
import os
import struct

import numpy as np

import mav1cu

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmav1.so")
CLI_PATH = os.path.join(HERE, "mav1enc")

EXPORTS = ["mav1_default_config", "mav1_create", "mav1_encode", "mav1_send_frame", "mav1_receive_packet",
           "mav1_receive_packet_wait", "mav1_pending_packets", "mav1_busy", "mav1_sequence_header", "mav1_get_recon",
           "mav1_last_stats", "mav1_backend_name", "mav1_tool_names", "mav1_destroy",
           # include/mav1_cuda.h
           "mav1_cuda_get_counters", "mav1_cuda_device_bytes", "mav1_cuda_device_bytes_for", "mav1_cuda_restart"]


class FrameStats(ctypes.Structure):
    """Mav1FrameStats (src/mav1.h:44-50)."""
    _fields_ = [("frame_type", ctypes.c_int), ("bytes", ctypes.c_size_t), ("num_blocks", ctypes.c_int),
                ("num_inter_blocks", ctypes.c_int), ("tool_use", ctypes.c_int * 16), ("t_analysis", ctypes.c_double),
                ("t_recon", ctypes.c_double), ("t_filter", ctypes.c_double), ("t_entropy", ctypes.c_double)]


class Counters(ctypes.Structure):
    """mav1_cuda_counters (include/mav1_cuda.h)."""
    _fields_ = [("frames", ctypes.c_int64), ("h2d_bytes", ctypes.c_int64), ("d2h_bytes", ctypes.c_int64),
                ("entropy_s", ctypes.c_double)]


_lib = None
_libc = ctypes.CDLL(None)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libmav1.so not built at {LIB_PATH}: run __graft_entry__.build()")
        mav1cu.lib()  # libmav1cu.so first (libmav1.so links it)
        L = ctypes.CDLL(LIB_PATH)
        vp, sz, i32 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int
        L.mav1_default_config.argtypes = [vp, i32, i32]
        L.mav1_default_config.restype = None
        L.mav1_create.argtypes = [vp, ctypes.c_char_p, sz]
        L.mav1_create.restype = vp
        L.mav1_send_frame.argtypes = [vp, vp, vp]
        L.mav1_send_frame.restype = i32
        L.mav1_receive_packet.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(sz)]
        L.mav1_receive_packet.restype = i32
        L.mav1_receive_packet_wait.argtypes = [vp, ctypes.POINTER(vp), ctypes.POINTER(sz), i32]
        L.mav1_receive_packet_wait.restype = i32
        L.mav1_pending_packets.argtypes = [vp]
        L.mav1_busy.argtypes = [vp]
        L.mav1_get_recon.argtypes = [vp, vp, vp]
        L.mav1_get_recon.restype = None
        L.mav1_last_stats.argtypes = [vp]
        L.mav1_last_stats.restype = ctypes.POINTER(FrameStats)
        L.mav1_backend_name.argtypes = [vp]
        L.mav1_backend_name.restype = ctypes.c_char_p
        L.mav1_sequence_header.argtypes = [vp, vp]
        L.mav1_sequence_header.restype = sz
        L.mav1_destroy.argtypes = [vp]
        L.mav1_destroy.restype = None
        L.mav1_cuda_get_counters.argtypes = [vp, ctypes.POINTER(Counters)]
        L.mav1_cuda_get_counters.restype = None
        L.mav1_cuda_device_bytes.argtypes = [vp]
        L.mav1_cuda_device_bytes.restype = ctypes.c_int64
        L.mav1_cuda_device_bytes_for.argtypes = [vp]
        L.mav1_cuda_device_bytes_for.restype = ctypes.c_int64
        L.mav1_cuda_restart.argtypes = [vp, vp]
        L.mav1_cuda_restart.restype = i32
        _libc.free.argtypes = [vp]
        _lib = L
    return _lib


class Mav1Error(RuntimeError):
    pass


class Encoder:
    """One mav1 encoder (Mav1Encoder) on the current CUDA device.

    cfg: a mav1cu.cli_config(...) record (the byte layout of Mav1Config)."""

    def __init__(self, cfg):
        self.lib = lib()
        self.cfg = np.ascontiguousarray(cfg)
        c = self.cfg[0]
        self.w, self.h = int(c["width"]), int(c["height"])
        self.cw, self.ch = (self.w + 1) // 2, (self.h + 1) // 2
        err = ctypes.create_string_buffer(512)
        self.h_ = self.lib.mav1_create(self.cfg.ctypes.data, err, 512)
        if not self.h_:
            raise Mav1Error("mav1_create: " + err.value.decode())
        self._strides = (ctypes.c_int * 3)(self.w, self.cw, self.cw)

    def send(self, i420):
        """Queues one frame: packed I420 bytes (numpy uint8), or None to flush."""
        if i420 is None:
            rc = self.lib.mav1_send_frame(self.h_, None, None)
        else:
            if isinstance(i420, (bytes, bytearray, memoryview)):
                i420 = np.frombuffer(i420, np.uint8)
            a = np.ascontiguousarray(i420, np.uint8).reshape(-1)
            if a.size != self.w * self.h + 2 * self.cw * self.ch:
                raise Mav1Error(f"frame of {a.size} bytes, expected {self.w * self.h + 2 * self.cw * self.ch}")
            y = self.w * self.h
            c = self.cw * self.ch
            base = a.ctypes.data
            ptrs = (ctypes.c_void_p * 3)(base, base + y, base + y + c)
            rc = self.lib.mav1_send_frame(self.h_, ptrs, self._strides)
        if rc:
            raise Mav1Error(f"mav1_send_frame failed ({rc})")

    def receive(self, recon=True, wait_ms=None):
        """Next temporal unit as (bytes, reconstruction or None), or None."""
        pkt, n = ctypes.c_void_p(), ctypes.c_size_t()
        if wait_ms is None:
            rc = self.lib.mav1_receive_packet(self.h_, ctypes.byref(pkt), ctypes.byref(n))
        else:
            rc = self.lib.mav1_receive_packet_wait(self.h_, ctypes.byref(pkt), ctypes.byref(n), wait_ms)
        if rc:
            return None
        data = ctypes.string_at(pkt, n.value)
        _libc.free(pkt)
        rec = self.recon() if recon else None
        return data, rec

    def recon(self):
        rec = [np.zeros((self.h, self.w), np.uint8), np.zeros((self.ch, self.cw), np.uint8),
               np.zeros((self.ch, self.cw), np.uint8)]
        ptrs = (ctypes.c_void_p * 3)(*[a.ctypes.data for a in rec])
        self.lib.mav1_get_recon(self.h_, ptrs, self._strides)
        return rec

    def stats(self):
        return self.lib.mav1_last_stats(self.h_).contents

    def counters(self):
        c = Counters()
        self.lib.mav1_cuda_get_counters(self.h_, ctypes.byref(c))
        return c

    def busy(self):
        return self.lib.mav1_busy(self.h_)

    def device_bytes(self):
        return self.lib.mav1_cuda_device_bytes(self.h_)

    def restart(self, cfg):
        """A new clip on this encoder (same frame size; device memory kept)."""
        cfg = np.ascontiguousarray(cfg)
        if self.lib.mav1_cuda_restart(self.h_, cfg.ctypes.data):
            raise Mav1Error("mav1_cuda_restart failed")
        self.cfg = cfg

    def close(self):
        if self.h_:
            self.lib.mav1_destroy(self.h_)
            self.h_ = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def encode(frames, cfg, recon=True, counters=None):
    """The clip through the queue API like tools/mav1enc.c: after every sent
    frame, the packets ready so far; then a flush. frames: packed I420 arrays.
    Returns (packets, reconstructions); counters (a list) receives the
    encoder's mav1_cuda_counters."""
    enc = Encoder(cfg)
    packets, recons = [], []
    try:
        for f in list(frames) + [None]:
            enc.send(f)
            while True:
                r = enc.receive(recon)
                if r is None:
                    break
                packets.append(r[0])
                recons.append(r[1])
        if counters is not None:
            counters.append(enc.counters())
    finally:
        enc.close()
    return packets, recons


def device_bytes_for(cfg):
    """Device bytes mav1_create would allocate for the configuration."""
    return lib().mav1_cuda_device_bytes_for(np.ascontiguousarray(cfg).ctypes.data)


def code_frames(enc, frames, expect, recon=True, timeout_ms=60000):
    """Sends frames to a live encoder (no flush) and receives `expect`
    temporal units: the ones ready after each send, then the rest as they
    complete. With closed GOPs (the frames start at a key frame and end at
    the next key-frame boundary), every frame's temporal unit comes out
    without a flush, so one encoder can code clip after clip. Returns
    (packets, reconstructions)."""
    packets, recons = [], []

    def drain(wait):
        while len(packets) < expect:
            r = enc.receive(recon, wait_ms=timeout_ms if wait else None)
            if r is None:
                if wait:
                    raise Mav1Error(f"no temporal unit within {timeout_ms} ms ({len(packets)} of {expect})")
                return
            packets.append(r[0])
            recons.append(r[1])

    for f in frames:
        enc.send(f)
        drain(False)
    drain(True)
    return packets, recons


def ivf_bytes(packets, w, h, fps=(30, 1)):
    """IVF container as tools/mav1enc.c writes it: the 32-byte file header
    (frame count patched in), then per temporal unit its size, its index as
    the timestamp and its bytes."""
    out = bytearray(b"DKIF" + struct.pack("<HH4sHHIIII", 0, 32, b"AV01", w, h, fps[0], fps[1], len(packets), 0))
    for i, p in enumerate(packets):
        out += struct.pack("<IQ", len(p), i) + p
    return bytes(out)
