"""Python binding of libmav1cu (include/mav1cu.h) over ctypes.

This is the host-side mirror of the encoder's backend interface for tests,
benchmarks and the batching / serving layers: a Session owns one encoder
instance's device state; its methods are the C ABI's stage calls. Record
formats (FrameParams, BlockInfo, SbInfo, LrUnit) are exposed as numpy dtypes
with the reference encoder's byte layout.

The CUDA library is required: importing this module on a machine where
libmav1cu.so is absent or cannot be loaded raises, there is no CPU fallback.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmav1cu.so")

# buffer ids (include/mav1cu.h)
BUF = dict(
    SRC=0, REC=1, REF=2, GOLD=3, PARAMS=4, MATS=5, MVFIELD=6, MVGOLD=7, BLOCKS=8, SBS=9, COEFS=10, LFMASK=11,
    CDEFBUF=12, CDEF_CHOICE=13, DBK=14, LROUT=15, LRUNITS=16, ACOSTS=17, AINFOS=18,
)

PARAM_FIELDS = [
    ("mi_cols", 1), ("mi_rows", 1), ("sb_cols", 1), ("sb_rows", 1), ("plane_w", 3), ("plane_h", 3), ("stride", 3),
    ("offset", 3), ("base_q_idx", 1), ("dc_q", 3), ("ac_q", 3), ("frame_is_intra", 1), ("reduced_tx_set", 1),
    ("enable_intra_edge_filter", 1), ("tx_search", 1), ("lambda", 1), ("wave", 1), ("num_blocks", 1),
    ("frame_w", 1), ("frame_h", 1), ("me_range", 1), ("lossless", 1), ("tx_mode_select", 1), ("tile_w_sb", 1),
    ("fast", 1), ("leaf", 1), ("depth_thr", 1), ("switchable_interp", 1), ("golden", 1), ("ref2_frame", 1),
    ("compound", 1), ("lf_level", 4), ("lf_sharpness", 1), ("cdef_damping", 1), ("cdef_bits", 1),
    ("cdef_y_pri", 8), ("cdef_y_sec", 8), ("cdef_uv_pri", 8), ("cdef_uv_sec", 8), ("lr_type", 3),
    ("lr_unit_size", 3), ("lr_unit_rows", 3), ("lr_unit_cols", 3), ("lr_unit_off", 3), ("turbo", 1),
]
PARAMS_DTYPE = np.dtype([(n, "<i4", (k,)) if k > 1 else (n, "<i4") for n, k in PARAM_FIELDS])
BLOCK_DTYPE = np.dtype([
    ("mi_row", "<i4"), ("mi_col", "<i4"), ("bsize", "<i4"), ("is_inter", "<i4"), ("y_mode", "<i4"),
    ("uv_mode", "<i4"), ("angle_y", "<i4"), ("angle_uv", "<i4"), ("mv_row", "<i4"), ("mv_col", "<i4"),
    ("tx_type", "<i4"), ("eob", "<i4", (3,)), ("coef_off", "<i4", (3,)), ("cfl_alpha_u", "<i4"),
    ("cfl_alpha_v", "<i4"), ("tx_depth", "<i4"), ("tx_types_lo", "<i4"), ("tx_types_hi", "<i4"),
    ("interp_filter", "<i4"), ("ref_frame", "<i4"), ("ref_frame1", "<i4"), ("mv1_row", "<i4"), ("mv1_col", "<i4"),
])
SB_DTYPE = np.dtype([("first_block", "<i4"), ("num_blocks", "<i4"), ("sb_row", "<i4"), ("sb_col", "<i4"),
                     ("part", "<i4", (85,))])
LRUNIT_DTYPE = np.dtype([("type", "<i4"), ("set", "<i4"), ("xqd", "<i4", (2,)), ("wiener", "<i4", (2, 3)),
                         ("pad", "<i4", (2,))])
CONFIG_FIELDS = ["width", "height", "qindex", "use_metal", "keyint", "tx_search", "tx_depth", "loop_filter", "cdef",
                 "restoration", "tile_cols_log2", "intra_edge_filter", "nonref_odd", "fast", "multi_ref", "altref",
                 "leaf", "switchable_interp", "lr_test", "me_range", "threads", "turbo"]
CONFIG_DTYPE = np.dtype([(n, "<i4") for n in CONFIG_FIELDS])
JOB_DTYPE = np.dtype([(n, "<i4") for n in [
    "disp", "is_key", "kind", "last_slot", "arf_slot", "refresh", "hidden", "base_q_idx", "order_hint", "nonref",
    "leafopt", "reference_select", "golden_refresh", "gold_differs", "show_existing", "pad"]])
assert PARAMS_DTYPE.itemsize == 392 and BLOCK_DTYPE.itemsize == 108
EXPORT_HEADER_DTYPE = np.dtype([
    ("status", "<i4"), ("seq", "<i4"), ("num_sbs", "<i4"), ("num_blocks", "<i4"), ("num_coefs", "<i4"),
    ("zero_run", "<i4"), ("sbs_off", "<i8"), ("cdef_off", "<i8"), ("blocks_off", "<i8"), ("coefs_off", "<i8"),
    ("rec_off", "<i8"), ("rec_bytes", "<i8"), ("bytes", "<i8"), ("params_off", "<i8"), ("lr_off", "<i8"),
    ("lr_units", "<i4"), ("pad", "<i4")])
EXPORT_REC = 1
EXPORT_LR = 2
assert SB_DTYPE.itemsize == 356 and LRUNIT_DTYPE.itemsize == 48 and EXPORT_HEADER_DTYPE.itemsize == 104

EXPORTS = [
    "mav1cu_session_create", "mav1cu_session_destroy", "mav1cu_set_stream", "mav1cu_get_stream", "mav1cu_buf_size",
    "mav1cu_buf_device", "mav1cu_upload", "mav1cu_download", "mav1cu_copy", "mav1cu_set_params",
    "mav1cu_motion_search", "mav1cu_analyze", "mav1cu_edge_types", "mav1cu_recon", "mav1cu_frame_core",
    "mav1cu_filter_info", "mav1cu_filter", "mav1cu_cdef_select", "mav1cu_restore", "mav1cu_synchronize",
    "mav1cu_error_string", "mav1cu_launch_count", "mav1cu_build_fwd_matrices", "mav1cu_plan",
    "mav1cu_frame_params_for", "mav1cu_stream_create", "mav1cu_stream_destroy", "mav1cu_stream_session",
    "mav1cu_stream_encode", "mav1cu_stream_slot", "mav1cu_stream_engines", "mav1cu_stream_engine",
    "mav1cu_stream_wait", "mav1cu_stream_join", "mav1cu_stream_synchronize", "mav1cu_edge_types_noalloc",
    "mav1cu_export_capacity", "mav1cu_export_image", "mav1cu_export", "mav1cu_lr_search", "mav1cu_plan_frames",
    "mav1cu_layout_of", "mav1cu_export_seq", "mav1cu_export_wait", "mav1cu_export_query", "mav1cu_host_alloc",
    "mav1cu_host_free", "mav1cu_debug_recon_fault", "mav1cu_stream_reconfigure", "mav1cu_stream_device_bytes", "mav1cu_stream_bytes_for", "mav1cu_session_device_bytes",
]


def load_library(path=LIB_PATH):
    """Loads libmav1cu.so and declares its signatures; raises if missing."""
    if not os.path.exists(path):
        raise RuntimeError(f"libmav1cu.so not built at {path}: run __graft_entry__.build()")
    lib = ctypes.CDLL(path)
    vp, sz, i32 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int
    lib.mav1cu_session_create.argtypes = [i32, i32, i32, ctypes.POINTER(vp), ctypes.c_char_p, sz]
    lib.mav1cu_session_create.restype = i32
    lib.mav1cu_session_destroy.argtypes = [vp]
    lib.mav1cu_session_destroy.restype = None
    lib.mav1cu_set_stream.argtypes = [vp, vp]
    lib.mav1cu_get_stream.argtypes = [vp]
    lib.mav1cu_get_stream.restype = vp
    lib.mav1cu_buf_size.argtypes = [vp, i32]
    lib.mav1cu_buf_size.restype = sz
    lib.mav1cu_buf_device.argtypes = [vp, i32]
    lib.mav1cu_buf_device.restype = vp
    for f in ("mav1cu_upload", "mav1cu_download"):
        getattr(lib, f).argtypes = [vp, i32, vp, sz]
        getattr(lib, f).restype = i32
    lib.mav1cu_copy.argtypes = [vp, i32, i32, sz]
    lib.mav1cu_set_params.argtypes = [vp, vp]
    for f in ("mav1cu_motion_search", "mav1cu_analyze", "mav1cu_edge_types", "mav1cu_recon", "mav1cu_frame_core",
              "mav1cu_filter_info", "mav1cu_restore", "mav1cu_synchronize"):
        getattr(lib, f).argtypes = [vp]
        getattr(lib, f).restype = i32
    lib.mav1cu_filter.argtypes = [vp, i32]
    lib.mav1cu_debug_recon_fault.argtypes = [vp, i32, i32]
    lib.mav1cu_debug_recon_fault.restype = i32
    lib.mav1cu_lr_search.argtypes = [vp, i32]
    lib.mav1cu_lr_search.restype = i32
    lib.mav1cu_cdef_select.argtypes = [vp, i32]
    lib.mav1cu_error_string.argtypes = [vp]
    lib.mav1cu_error_string.restype = ctypes.c_char_p
    lib.mav1cu_launch_count.argtypes = [vp]
    lib.mav1cu_launch_count.restype = ctypes.c_int64
    lib.mav1cu_build_fwd_matrices.argtypes = [vp]
    lib.mav1cu_build_fwd_matrices.restype = None
    lib.mav1cu_plan.argtypes = [vp, i32, vp, i32]
    lib.mav1cu_plan.restype = i32
    lib.mav1cu_frame_params_for.argtypes = [vp, vp, vp, ctypes.POINTER(i32)]
    lib.mav1cu_frame_params_for.restype = i32
    lib.mav1cu_stream_create.argtypes = [vp, ctypes.POINTER(vp), ctypes.c_char_p, sz]
    lib.mav1cu_stream_create.restype = i32
    lib.mav1cu_stream_destroy.argtypes = [vp]
    lib.mav1cu_stream_destroy.restype = None
    lib.mav1cu_stream_session.argtypes = [vp]
    lib.mav1cu_stream_session.restype = vp
    lib.mav1cu_stream_encode.argtypes = [vp, vp, vp, i32]
    lib.mav1cu_stream_encode.restype = i32
    lib.mav1cu_stream_slot.argtypes = [vp, i32]
    lib.mav1cu_stream_slot.restype = vp
    lib.mav1cu_stream_engines.argtypes = [vp]
    lib.mav1cu_stream_engines.restype = i32
    lib.mav1cu_stream_engine.argtypes = [vp, i32]
    lib.mav1cu_stream_engine.restype = vp
    for f in ("mav1cu_stream_wait", "mav1cu_stream_join"):
        getattr(lib, f).argtypes = [vp, vp]
        getattr(lib, f).restype = i32
    lib.mav1cu_stream_synchronize.argtypes = [vp]
    lib.mav1cu_stream_synchronize.restype = i32
    lib.mav1cu_edge_types_noalloc.argtypes = [vp, vp, vp, i32, i32, i32, vp, ctypes.c_char_p, sz]
    lib.mav1cu_edge_types_noalloc.restype = i32
    lib.mav1cu_export_capacity.argtypes = [vp]
    lib.mav1cu_export_capacity.restype = sz
    lib.mav1cu_export_image.argtypes = [vp]
    lib.mav1cu_export_image.restype = vp
    lib.mav1cu_export.argtypes = [vp, vp, sz, i32]
    lib.mav1cu_export.restype = i32
    return lib


COUNT_LIB_PATH = os.path.join(HERE, "libmav1cu_count.so")
# the counting build's categories (include/mav1cu_count.h), in counter order
WORK_NAMES = ["me_sad", "me_dec_sad", "me_satd", "qpel_taps", "ana_satd", "ana_inter_px", "ana_intra_px", "ana_cfl",
              "rec_inter_px", "rec_intra_px", "fwd_mac", "quant", "inv_ops", "lf_taps", "cdef_taps", "lr_taps"]


def load_count_library(path=COUNT_LIB_PATH):
    """libmav1cu_count.so (every mav1cu entry point plus the work counters);
    raises if it is missing."""
    lib_ = load_library(path)
    lib_.mav1cu_work_read.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib_.mav1cu_work_read.restype = ctypes.c_int
    lib_.mav1cu_work_reset.argtypes = []
    lib_.mav1cu_work_reset.restype = ctypes.c_int
    lib_.mav1cu_work_int_peak.argtypes = [ctypes.POINTER(ctypes.c_double)]
    lib_.mav1cu_work_int_peak.restype = ctypes.c_int
    return lib_


def work_read(lib_):
    """The counters of the counting build as {category: units}."""
    v = np.zeros(len(WORK_NAMES), np.uint64)
    rc = lib_.mav1cu_work_read(v.ctypes.data, len(WORK_NAMES))
    if rc != len(WORK_NAMES):
        raise Mav1cuError(f"mav1cu_work_read: {rc}")
    return dict(zip(WORK_NAMES, (int(x) for x in v)))


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = load_library()
    return _lib


class Mav1cuError(RuntimeError):
    pass


def geometry(width, height):
    """Frame layout of the reference encoder (encoder.c:93-120)."""
    mi_cols, mi_rows = 2 * ((width + 7) >> 3), 2 * ((height + 7) >> 3)
    sb_cols, sb_rows = (mi_cols + 15) >> 4, (mi_rows + 15) >> 4
    stride = [sb_cols * 64, sb_cols * 32, sb_cols * 32]
    plane_h = [sb_rows * 64, sb_rows * 32, sb_rows * 32]
    offset = [0, stride[0] * plane_h[0], stride[0] * plane_h[0] + stride[1] * plane_h[1]]
    return dict(w=width, h=height, mi_cols=mi_cols, mi_rows=mi_rows, sb_cols=sb_cols, sb_rows=sb_rows,
                num_sbs=sb_cols * sb_rows, stride=stride, plane_h=plane_h, offset=offset,
                frame_bytes=offset[2] + stride[2] * plane_h[2])


def fwd_matrices():
    m = np.zeros(15 * 4096, np.int32)
    lib().mav1cu_build_fwd_matrices(m.ctypes.data)
    return m


class Session:
    """Device state of one encoder instance (mav1cu_session)."""

    def __init__(self, width, height, max_cdef_presets=4):
        self.lib = lib()
        self.geom = geometry(width, height)
        h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        rc = self.lib.mav1cu_session_create(width, height, max_cdef_presets, ctypes.byref(h), err, 512)
        if rc != 0:
            raise Mav1cuError(f"mav1cu_session_create: {err.value.decode()} ({rc})")
        self.h = h

    def close(self):
        if self.h:
            self.lib.mav1cu_session_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc, what):
        if rc != 0:
            raise Mav1cuError(f"{what}: {self.lib.mav1cu_error_string(self.h).decode()} ({rc})")

    def size(self, buf):
        return self.lib.mav1cu_buf_size(self.h, BUF[buf])

    def device_ptr(self, buf):
        return self.lib.mav1cu_buf_device(self.h, BUF[buf])

    def set_stream(self, stream_ptr):
        self.lib.mav1cu_set_stream(self.h, stream_ptr)

    def upload(self, buf, arr):
        arr = np.ascontiguousarray(arr)
        self._check(self.lib.mav1cu_upload(self.h, BUF[buf], arr.ctypes.data, arr.nbytes), f"upload {buf}")

    def download(self, buf, dtype=np.uint8, count=None, out=None):
        if out is None:
            n = self.size(buf) // np.dtype(dtype).itemsize if count is None else count
            out = np.empty(n, dtype)
        self._check(self.lib.mav1cu_download(self.h, BUF[buf], out.ctypes.data, out.nbytes), f"download {buf}")
        self.synchronize()
        return out

    def copy(self, dst, src, nbytes=None):
        n = min(self.size(dst), self.size(src)) if nbytes is None else nbytes
        self._check(self.lib.mav1cu_copy(self.h, BUF[dst], BUF[src], n), "copy")

    def set_params(self, params):
        p = np.ascontiguousarray(params)
        assert p.nbytes == 392
        self._check(self.lib.mav1cu_set_params(self.h, p.ctypes.data), "set_params")

    def motion_search(self):
        self._check(self.lib.mav1cu_motion_search(self.h), "motion_search")

    def analyze(self):
        self._check(self.lib.mav1cu_analyze(self.h), "analyze")

    def edge_types(self):
        self._check(self.lib.mav1cu_edge_types(self.h), "edge_types")

    def recon(self):
        self._check(self.lib.mav1cu_recon(self.h), "recon")

    def frame_core(self):
        self._check(self.lib.mav1cu_frame_core(self.h), "frame_core")

    def filter_info(self):
        self._check(self.lib.mav1cu_filter_info(self.h), "filter_info")

    def filter(self, num_cdef_presets):
        self._check(self.lib.mav1cu_filter(self.h, num_cdef_presets), "filter")

    def cdef_select(self, num_cdef_presets):
        self._check(self.lib.mav1cu_cdef_select(self.h, num_cdef_presets), "cdef_select")

    def restore(self):
        self._check(self.lib.mav1cu_restore(self.h), "restore")

    def lr_search(self, lr_test=0):
        self._check(self.lib.mav1cu_lr_search(self.h, lr_test), "lr_search")

    def synchronize(self):
        self._check(self.lib.mav1cu_synchronize(self.h), "synchronize")

    def export_capacity(self):
        return self.lib.mav1cu_export_capacity(self.h)

    def export(self, image_ptr=None, cap=None, rec=False):
        """Enqueues the compact export of the writer inputs (and with rec the
        shown reconstruction) into image_ptr (mapped page-locked host or
        device memory), or into the session's own image; returns the image's
        address."""
        if image_ptr is None:
            image_ptr = self.lib.mav1cu_export_image(self.h)
            if not image_ptr:
                self._check(-2, "export image")
        cap = self.export_capacity() if cap is None else cap
        self._check(self.lib.mav1cu_export(self.h, image_ptr, cap, EXPORT_REC if rec else 0), "export")
        return image_ptr

    def launches(self):
        return self.lib.mav1cu_launch_count(self.h)


def export_sections(image):
    """(header, superblocks, CDEF choices, blocks, levels, reconstruction) of
    an export image held in a uint8 array (reconstruction: None when the
    export left it out)."""
    h = image[:EXPORT_HEADER_DTYPE.itemsize].view(EXPORT_HEADER_DTYPE)[0]
    if h["status"]:
        raise Mav1cuError(f"export image status {int(h['status'])}")
    nsb, nb, nc = int(h["num_sbs"]), int(h["num_blocks"]), int(h["num_coefs"])

    def sect(off, dtype, n):
        return image[int(off):int(off) + n * np.dtype(dtype).itemsize].view(dtype)

    rec = sect(h["rec_off"], np.uint8, int(h["rec_bytes"])) if h["rec_bytes"] else None
    return (h, sect(h["sbs_off"], SB_DTYPE, nsb), sect(h["cdef_off"], np.int8, nsb),
            sect(h["blocks_off"], BLOCK_DTYPE, nb), sect(h["coefs_off"], np.int32, nc), rec)


def cli_config(width, height, q=100, keyint=0, lf=1, cdef=1, txs=1, txd=1, lr=1, lr_test=0, sw=1, fast=0, turbo=0,
               golden=0, altref=0, leaf=0, edge=1, tiles=-1, me_range=32):
    """mav1cu_config as the reference CLI (tools/mav1enc.c:36-104) builds its
    Mav1Config from the same flags (defaults of mav1_default_config)."""
    c = np.zeros(1, CONFIG_DTYPE)[0]
    if turbo:
        fast = 1
    vals = dict(width=width, height=height, qindex=q, use_metal=1, keyint=keyint, tx_search=txs, tx_depth=txd,
                loop_filter=lf, cdef=cdef, restoration=lr, lr_test=lr_test, switchable_interp=sw, me_range=me_range,
                fast=fast, turbo=turbo, multi_ref=golden, altref=altref, leaf=leaf, nonref_odd=0,
                intra_edge_filter=edge, tile_cols_log2=tiles if tiles >= 0 else (2 if turbo else 3 if fast else 0))
    for k, v in vals.items():
        c[k] = v
    if fast:
        c["tx_search"] = c["tx_depth"] = c["restoration"] = c["switchable_interp"] = 0
    return np.array([c], CONFIG_DTYPE)


def plan(cfg, nframes):
    """Coding order of a clip (mav1cu_plan): structured array of jobs."""
    jobs = np.zeros(4 * nframes + 8, JOB_DTYPE)
    n = lib().mav1cu_plan(cfg.ctypes.data, nframes, jobs.ctypes.data, len(jobs))
    if n < 0:
        raise Mav1cuError(f"mav1cu_plan: {n}")
    return jobs[:n]


def frame_params(cfg, job):
    """(FrameParams as 392 raw bytes, CDEF presets the filter stage writes)."""
    fp = np.zeros(392, np.uint8)
    presets = ctypes.c_int()
    j = np.array([job], JOB_DTYPE)
    rc = lib().mav1cu_frame_params_for(cfg.ctypes.data, j.ctypes.data, fp.ctypes.data, ctypes.byref(presets))
    if rc:
        raise Mav1cuError(f"mav1cu_frame_params_for: {rc}")
    return fp, presets.value


class _EngineSession(Session):
    """A session owned by a stream (not closed by Python)."""

    def __init__(self, lib_, ptr, geom):
        self.lib, self.h, self.geom = lib_, ctypes.c_void_p(ptr), geom

    def close(self):
        pass


class Stream:
    """Device-resident stream (mav1cu_stream): planned frames coded through
    every device stage with the reference slots in HBM, reference-chain and
    non-reference frames on two concurrent engines."""

    def __init__(self, cfg):
        self.lib = lib()
        self.cfg = cfg
        h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(512)
        rc = self.lib.mav1cu_stream_create(cfg.ctypes.data, ctypes.byref(h), err, 512)
        if rc:
            raise Mav1cuError(f"mav1cu_stream_create: {err.value.decode()} ({rc})")
        self.h = h
        geom = geometry(int(cfg[0]["width"]), int(cfg[0]["height"]))
        self.engines = [_EngineSession(self.lib, self.lib.mav1cu_stream_engine(h, k), geom)
                        for k in range(self.lib.mav1cu_stream_engines(h))]
        self.session = self.engines[0]

    @staticmethod
    def engine_of(job):
        """Engine that codes the job: 0 for frames that refresh a slot, else 1."""
        return 0 if (job["is_key"] or job["refresh"]) else 1

    def encode(self, job, i420_ptr, on_device):
        """Enqueues one planned frame; returns the session holding its outputs."""
        j = np.array([job], JOB_DTYPE)
        rc = self.lib.mav1cu_stream_encode(self.h, j.ctypes.data, i420_ptr, 1 if on_device else 0)
        e = self.engines[self.engine_of(job)]
        if rc:
            raise Mav1cuError(f"mav1cu_stream_encode: {self.lib.mav1cu_error_string(e.h).decode()}")
        return e

    def wait(self, cuda_stream):
        self.lib.mav1cu_stream_wait(self.h, cuda_stream)

    def join(self, cuda_stream):
        self.lib.mav1cu_stream_join(self.h, cuda_stream)

    def synchronize(self):
        rc = self.lib.mav1cu_stream_synchronize(self.h)
        if rc:
            msgs = [self.lib.mav1cu_error_string(e.h).decode() for e in self.engines]
            raise Mav1cuError(f"stream: {msgs}")

    def launches(self):
        return sum(e.launches() for e in self.engines)

    def slot_ptr(self, k):
        return self.lib.mav1cu_stream_slot(self.h, k)

    def close(self):
        if self.h:
            self.lib.mav1cu_stream_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
