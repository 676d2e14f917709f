/*
 * mav1cu — B200 (sm_100a) encode backend for the mav1 AV1 encoder.
 *
 * C ABI of libmav1cu.so: plain pointers, sizes and status codes; no CUDA or
 * C++ types cross it (a CUDA stream is passed as void *). One session holds
 * the device-resident state of one encoder instance: its frame buffers,
 * reference pictures, analysis tables and stage outputs, laid out exactly as
 * the reference encoder's shared buffers so the host entropy coder reads
 * them unchanged.
 *
 * The stage entry points are the hooks of the reference's backend vtable
 * (src/backend.h:10-24 of neolite/mav1-encoder) plus the host helpers of its
 * frame driver that run on the device here; each cites the reference
 * function it replaces. Stage calls are asynchronous on the session's stream
 * and return MAV1CU_OK once enqueued; errors are sticky per session
 * (mav1cu_error_string) and reported by the next call.
 */
#ifndef MAV1CU_H
#define MAV1CU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- record formats shared with the host encoder ------------------------
 * Byte-identical to the reference's structs (the host tile writer reads
 * them): FrameParams src/kernels/k_common.h:52-85 (392 bytes), BlockInfo
 * k_common.h:98-120 (108 bytes), SbInfo k_common.h:123-128 (356 bytes),
 * LrUnit src/kernels/k_lr.h:12-18 (48 bytes). Every field is 32 bits. */
typedef struct {
  int32_t mi_cols, mi_rows;
  int32_t sb_cols, sb_rows;
  int32_t plane_w[3], plane_h[3];
  int32_t stride[3], offset[3];
  int32_t base_q_idx;
  int32_t dc_q[3], ac_q[3];
  int32_t frame_is_intra;
  int32_t reduced_tx_set;
  int32_t enable_intra_edge_filter;
  int32_t tx_search;
  int32_t lambda;
  int32_t wave;
  int32_t num_blocks;
  int32_t frame_w, frame_h;
  int32_t me_range;
  int32_t lossless;
  int32_t tx_mode_select;
  int32_t tile_w_sb;
  int32_t fast;
  int32_t leaf;
  int32_t depth_thr;
  int32_t switchable_interp;
  int32_t golden;
  int32_t ref2_frame;
  int32_t compound;
  int32_t lf_level[4];
  int32_t lf_sharpness;
  int32_t cdef_damping, cdef_bits;
  int32_t cdef_y_pri[8], cdef_y_sec[8], cdef_uv_pri[8], cdef_uv_sec[8];
  int32_t lr_type[3], lr_unit_size[3], lr_unit_rows[3], lr_unit_cols[3], lr_unit_off[3];
  int32_t turbo;
} mav1cu_frame_params;

typedef struct {
  int32_t mi_row, mi_col, bsize;
  int32_t is_inter;
  int32_t y_mode, uv_mode, angle_y, angle_uv;
  int32_t mv_row, mv_col;
  int32_t tx_type;
  int32_t eob[3];
  int32_t coef_off[3];
  int32_t cfl_alpha_u, cfl_alpha_v;
  int32_t tx_depth;
  int32_t tx_types_lo, tx_types_hi;
  int32_t interp_filter;
  int32_t ref_frame;
  int32_t ref_frame1;
  int32_t mv1_row, mv1_col;
} mav1cu_block_info;

typedef struct {
  int32_t first_block, num_blocks;
  int32_t sb_row, sb_col;
  int32_t part[85];
} mav1cu_sb_info;

typedef struct {
  int32_t type;
  int32_t set;
  int32_t xqd[2];
  int32_t wiener[2][3];
  int32_t pad[2];
} mav1cu_lr_unit;

/* ---- status codes -------------------------------------------------------- */
enum {
  MAV1CU_OK = 0,
  MAV1CU_ERR_ARG = -1,      /* bad argument (size, buffer id, state) */
  MAV1CU_ERR_CUDA = -2,     /* a CUDA runtime call failed (see mav1cu_error_string) */
  MAV1CU_ERR_NOMEM = -3,    /* device allocation failed */
  MAV1CU_ERR_DEVICE = -4,   /* a kernel reported an error through its status word */
};

/* ---- session buffers (the reference encoder's Bufs, enc_internal.h:81-151) */
enum {
  MAV1CU_BUF_SRC = 0,       /* padded source frame, frame_bytes (encoder.c:113-120,297-310) */
  MAV1CU_BUF_REC,           /* reconstruction, frame_bytes */
  MAV1CU_BUF_REF,           /* LAST reference picture, frame_bytes */
  MAV1CU_BUF_GOLD,          /* second reference (GOLDEN / ALTREF), frame_bytes */
  MAV1CU_BUF_PARAMS,        /* mav1cu_frame_params */
  MAV1CU_BUF_MATS,          /* forward matrices, 15 x 4096 int32 (fwd_matrices.c:57-65) */
  MAV1CU_BUF_MVFIELD,       /* int32 [num_sbs][85][2] motion vectors of LAST */
  MAV1CU_BUF_MVGOLD,        /* int32 [num_sbs][85][2] motion vectors of the second reference */
  MAV1CU_BUF_BLOCKS,        /* mav1cu_block_info [num_sbs][64] (decode order) */
  MAV1CU_BUF_SBS,           /* mav1cu_sb_info [num_sbs] */
  MAV1CU_BUF_COEFS,         /* int32 [num_sbs][6144] quantised levels */
  MAV1CU_BUF_LFMASK,        /* uint8 [mi_rows][mi_cols]: bsize | skip << 5 | tx_depth << 6 */
  MAV1CU_BUF_CDEFBUF,       /* num presets x frame_bytes: CDEF output of every preset */
  MAV1CU_BUF_CDEF_CHOICE,   /* int8 [num_sbs]: chosen CDEF preset */
  MAV1CU_BUF_DBK,           /* deblocked frame before CDEF, frame_bytes */
  MAV1CU_BUF_LROUT,         /* loop-restoration output, frame_bytes */
  MAV1CU_BUF_LRUNITS,       /* mav1cu_lr_unit [3 (sb_rows+1)(sb_cols+1)] */
  MAV1CU_BUF_ACOSTS,        /* int64 [num_sbs][85*13] analysis pass-1 costs */
  MAV1CU_BUF_AINFOS,        /* mav1cu_block_info [num_sbs][85*13] analysis pass-1 decisions */
  MAV1CU_BUF_COUNT
};

typedef struct mav1cu_session mav1cu_session;

/* Creates a session for frames of width x height on the current CUDA device,
 * with room for `max_cdef_presets` (0..4) CDEF outputs. Allocates all device
 * state once (sized like the reference encoder's buffers, encoder.c:124-166).
 * Replaces backend_metal_create (src/backend.h:37, backend_metal.m:576-610).
 * Returns MAV1CU_OK and *out, or an error code with a message in err. */
int mav1cu_session_create(int width, int height, int max_cdef_presets, mav1cu_session **out, char *err,
                          size_t errlen);
/* Frees every device resource (Backend.destroy, backend.h:20). */
void mav1cu_session_destroy(mav1cu_session *s);

/* The CUDA stream (cudaStream_t) the session enqueues on; NULL: its own. */
int mav1cu_set_stream(mav1cu_session *s, void *stream);
void *mav1cu_get_stream(mav1cu_session *s);

/* Size in bytes and device address of a session buffer. */
size_t mav1cu_buf_size(const mav1cu_session *s, int buf);
void *mav1cu_buf_device(mav1cu_session *s, int buf);
/* Asynchronous copies between host memory and a session buffer (pinned host
 * memory makes them truly asynchronous). bytes <= mav1cu_buf_size. */
int mav1cu_upload(mav1cu_session *s, int buf, const void *host, size_t bytes);
int mav1cu_download(mav1cu_session *s, int buf, void *host, size_t bytes);
/* Device-to-device copy between two session buffers (e.g. rec -> ref). */
int mav1cu_copy(mav1cu_session *s, int dst_buf, int src_buf, size_t bytes);

/* Sets the frame parameters of the next stages: a host copy is kept (launch
 * shapes depend on it) and the record is uploaded to MAV1CU_BUF_PARAMS. */
int mav1cu_set_params(mav1cu_session *s, const mav1cu_frame_params *fp);

/* ---- stages (enqueue on the session stream) ------------------------------ */
/* Motion search of every node of every superblock, all levels, for LAST and
 * (fp.golden) the second reference: quarter-pel / decimated planes, full-pel
 * search, sub-pel refinement. Writes MVFIELD / MVGOLD.
 * Replaces Backend.motion_search (backend.h:12; backend_cpu.c:23-56). */
int mav1cu_motion_search(mav1cu_session *s);
/* Mode and partition analysis: pass 1 over every candidate block, pass 2
 * partition decision and block emission. Writes ACOSTS, AINFOS, BLOCKS, SBS.
 * Replaces Backend.analyze (backend.h:13; backend_cpu.c:58-74). */
int mav1cu_analyze(mav1cu_session *s);
/* Intra edge filter types of every block into BlockInfo.interp_filter bits
 * 4/5. Replaces the host's edge_filter_types (encoder.c:319-346,399-404). */
int mav1cu_edge_types(mav1cu_session *s);
/* Reconstruction in decode order: prediction, forward transform,
 * quantisation, inverse transform. Writes REC, COEFS and the BlockInfo
 * recon fields. Replaces Backend.recon (backend.h:14; backend_cpu.c:76-156). */
int mav1cu_recon(mav1cu_session *s);
/* ME + analysis + edge types + recon of one frame (Backend.frame_core,
 * backend.h:21-23); motion search is skipped on intra frames. */
int mav1cu_frame_core(mav1cu_session *s);
/* Per-mi loop-filter info into LFMASK. Replaces build_filter_info
 * (encoder.c:513-526). */
int mav1cu_filter_info(mav1cu_session *s);
/* Deblocks REC in place, then writes CDEF output of presets 0..n-1 into
 * CDEFBUF (Backend.filter, backend.h:15-17; backend_cpu.c:158-177). */
int mav1cu_filter(mav1cu_session *s, int num_cdef_presets);
/* Picks every superblock's preset by SSE against SRC, writes CDEF_CHOICE and
 * copies the chosen output into REC. Replaces cdef_select (encoder.c:530-563). */
int mav1cu_cdef_select(mav1cu_session *s, int num_cdef_presets);
/* Loop restoration of REC (CDEF output) with DBK and LRUNITS into LROUT
 * (Backend.restore, backend.h:18-19; backend_cpu.c:179-188). */
int mav1cu_restore(mav1cu_session *s);
/* Loop-restoration parameter search: per restoration unit of every plane,
 * RESTORE_NONE, a least-squares Wiener filter with its greedy +-1 tap
 * refinement, or the best self-guided set with fitted projection weights, by
 * 16 * SSE + lambda * bits against SRC; from REC (CDEF output) and DBK (the
 * deblocked frame). Writes LRUNITS and lr_type of the device PARAMS record
 * (and of the next export's parameters section). lr_test: Mav1Config.lr_test
 * (Wiener on even units, the self-guided set of least SSE on odd ones).
 * Replaces lr_select (lr_search.c:244-359), a host step of the reference's
 * run_frame_core (encoder.c:636-638). */
int mav1cu_lr_search(mav1cu_session *s, int lr_test);

/* Failure detection without a device fault (a test hook): the session's next
 * mav1cu_recon counts one more luma dependency for intra block hold_block
 * than exists, so that block is never released, and its dependency waits
 * give up after spin_limit polls instead of about 2^22. The waiting workers
 * then set the session's device status and stop; the launch returns, the
 * context stays usable, and mav1cu_synchronize reports MAV1CU_ERR_DEVICE.
 * The session stays in error afterwards. No counterpart in the reference. */
int mav1cu_debug_recon_fault(mav1cu_session *s, int hold_block, int spin_limit);

/* Waits for the session stream; returns the sticky error state. */
int mav1cu_synchronize(mav1cu_session *s);
/* Message of the first error (empty string if none). */
const char *mav1cu_error_string(const mav1cu_session *s);
/* Number of kernel launches this session has enqueued since creation. */
int64_t mav1cu_launch_count(const mav1cu_session *s);


/* ---- encoder configuration and frame planning ---------------------------
 * mav1cu_config has the byte layout of the reference's Mav1Config
 * (src/mav1.h:20-42); the fields keep their meaning. */
typedef struct {
  int32_t width, height;
  int32_t qindex;
  int32_t use_metal;
  int32_t keyint;
  int32_t tx_search;
  int32_t tx_depth;
  int32_t loop_filter;
  int32_t cdef;
  int32_t restoration;
  int32_t tile_cols_log2;
  int32_t intra_edge_filter;
  int32_t nonref_odd;
  int32_t fast;
  int32_t multi_ref;
  int32_t altref;
  int32_t leaf;
  int32_t switchable_interp;
  int32_t lr_test;
  int32_t me_range;
  int32_t threads;
  int32_t turbo;
} mav1cu_config;

/* One coded frame of a stream, in coding order: the frame-structure
 * decisions of the reference's driver (mav1_encode, encoder.c:822-846, and
 * the ALTREF driver alt_drain / pyr_code / alt_code, encoder.c:1004-1293). */
typedef struct {
  int32_t disp;              /* display index of the source frame */
  int32_t is_key;
  int32_t kind;              /* 0 regular, 1 hidden ALTREF, 2 inside the mini-GOP, 3 pyramid middle */
  int32_t last_slot;         /* reference slot of LAST (-1: none) */
  int32_t arf_slot;          /* reference slot of the second reference (-1: none) */
  int32_t refresh;           /* refresh_frame_flags */
  int32_t hidden;            /* not shown (shown later by show_existing_frame) */
  int32_t base_q_idx;
  int32_t order_hint;
  int32_t nonref;            /* not kept as a reference */
  int32_t leafopt;           /* leaf-frame savings of this frame */
  int32_t reference_select;  /* compound LAST + ALTREF allowed */
  int32_t golden_refresh;    /* (no ALTREF) frame refreshes GOLDEN */
  int32_t gold_differs;      /* (no ALTREF) GOLDEN holds another frame than LAST */
  int32_t show_existing;     /* >= 0: after this frame a show_existing_frame of that slot follows */
  int32_t pad;
} mav1cu_frame_job;

/* Normalises cfg like the reference's encoder creation (turbo implies fast,
 * ALTREF >= 2 and leaf frames; encoder.c:69-90) and writes the coding order
 * of a clip of nframes frames into jobs (at most cap). Returns the number of
 * jobs, or a negative status. */
int mav1cu_plan(const mav1cu_config *cfg, int nframes, mav1cu_frame_job *jobs, int cap);
/* Incremental planning for a caller that receives frames one at a time (the
 * queue API mav1_send_frame, encoder.c:1295-1320): the state of the
 * reference driver's frame queue between calls. Zero-initialise it before the
 * first call. */
typedef struct {
  int32_t in_disp;        /* frames received so far */
  int32_t inq_n;          /* received frames not yet planned (ALTREF driver) */
  int32_t key_disp;       /* display index of the last key frame */
  int32_t anchor_slot;    /* slot of the last shown reference frame */
  int32_t ld_order_hint;  /* low-delay driver: OrderHint of the next frame */
  int32_t ld_last_id, ld_gold_id; /* low-delay driver: frames held by LAST / GOLDEN */
  int32_t pad[9];
} mav1cu_planner;

/* Adds new_frames received frames to the queue and writes the jobs that can
 * now be coded into jobs (coding order, at most cap): with ALTREF a mini-GOP
 * is planned once all of its frames are queued, or at once when flush is set
 * (end of stream: alt_drain, encoder.c:1252-1293); without ALTREF every frame
 * is planned as it arrives (mav1_encode, encoder.c:822-875). Returns the
 * number of jobs, or a negative status. The jobs of a whole clip equal
 * mav1cu_plan's, whatever the split into calls. */
int mav1cu_plan_frames(const mav1cu_config *cfg, mav1cu_planner *state, int new_frames, int flush,
                       mav1cu_frame_job *jobs, int cap);

/* Normalised configuration and tile geometry of an encoder (create_enc,
 * encoder.c:69-120): turbo implies fast, ALTREF >= 2 and leaf frames; the
 * tile columns are clamped to the frame. */
typedef struct {
  mav1cu_config cfg;      /* the normalised configuration */
  int32_t leafopt_cfg;    /* leaf-frame savings (MAV1_LEAFOPT, default 0x3F) */
  int32_t mi_cols, mi_rows, sb_cols, sb_rows, num_sbs;
  int32_t tile_cols_log2, tile_cols, tile_w_sb, min_log2_tile_cols, max_log2_tile_cols;
  int32_t stride[3], offset[3], plane_h[3];
  int64_t frame_bytes;
} mav1cu_layout;
int mav1cu_layout_of(const mav1cu_config *cfg, mav1cu_layout *out);

/* Frame parameters of one planned frame (setup_params, encoder.c:407-510).
 * *num_cdef_presets receives the presets the filter stage writes (0 with
 * CDEF off for the frame). */
int mav1cu_frame_params_for(const mav1cu_config *cfg, const mav1cu_frame_job *job, mav1cu_frame_params *fp,
                            int *num_cdef_presets);

/* A device-resident stream: one session plus the reference slots (8 frame
 * buffers in HBM); each call codes one planned frame through every device
 * stage (source load with edge replication, frame core, filter info,
 * deblocking, CDEF, CDEF selection, slot refresh). The frame's writer inputs
 * (BLOCKS, SBS, COEFS, CDEF_CHOICE, PARAMS) and its reconstruction (REC) are
 * in the session's buffers when the call's work completes. */
typedef struct mav1cu_stream mav1cu_stream;
int mav1cu_stream_create(const mav1cu_config *cfg, mav1cu_stream **out, char *err, size_t errlen);
void mav1cu_stream_destroy(mav1cu_stream *st);
mav1cu_session *mav1cu_stream_session(mav1cu_stream *st);
/* i420: packed I420 source of the job's frame (width x height luma, then the
 * two (w+1)/2 x (h+1)/2 chroma planes), in device memory if on_device, else
 * in host memory (pinned for an asynchronous copy). */
int mav1cu_stream_encode(mav1cu_stream *st, const mav1cu_frame_job *job, const void *i420, int on_device);
/* Device address of reference slot k (0..7), frame_bytes each. */
void *mav1cu_stream_slot(mav1cu_stream *st, int k);
/* Frame engines: the stream codes reference-chain frames (key, ALTREF,
 * regular: they refresh a slot) on engine 0 and non-reference frames on
 * engine 1, concurrently where the slot dependencies allow. Each engine is a
 * session with its own CUDA stream; a frame's outputs stay in its engine's
 * session buffers until that engine codes its next frame, and work the
 * caller enqueues on that session (mav1cu_download) is ordered after it.
 * mav1cu_stream_session returns the engine of the last encoded frame. */
int mav1cu_stream_engines(const mav1cu_stream *st);
mav1cu_session *mav1cu_stream_engine(mav1cu_stream *st, int k);
/* Every engine waits for the work enqueued on `stream` so far (wait), or
 * `stream` waits for every engine's work so far (join): brackets for timing
 * or ordering against other device work. */
int mav1cu_stream_wait(mav1cu_stream *st, void *stream);
int mav1cu_stream_join(mav1cu_stream *st, void *stream);
/* Waits for every engine; returns the first sticky error. */
int mav1cu_stream_synchronize(mav1cu_stream *st);
/* Starts a new clip on an existing stream (its device memory reused): waits
 * for its work, takes cfg (same width and height; the other settings may
 * change) and forgets the slot history. The next frame must be a key frame.
 * No counterpart in the reference, whose encoders code one clip each. */
int mav1cu_stream_reconfigure(mav1cu_stream *st, const mav1cu_config *cfg);
/* Device memory of a stream: what its engines and slots allocated (requested
 * bytes), and the same figure for a configuration before creating it (for
 * admission against a memory budget). */
int64_t mav1cu_stream_device_bytes(const mav1cu_stream *st);
int64_t mav1cu_stream_bytes_for(const mav1cu_config *cfg);
int64_t mav1cu_session_device_bytes(const mav1cu_session *s);

/* ---- compact export of the writer inputs ---------------------------------
 * No counterpart in the reference: its Metal backend shares full-size
 * buffers with the host (unified memory). Here the entropy coder's inputs
 * cross PCIe, so the device packs them into one image first:
 *   superblock table  num_sbs records; first_block rewritten to the packed
 *                     blocks (the only way the reference's host steps reach
 *                     blocks: tile_writer.c:585, encoder.c:327-337,519,678,717)
 *   CDEF choices      num_sbs int8
 *   blocks            the num_blocks records in use, superblock order;
 *                     coef_off[] rewritten into the level section
 *   levels            a run of zero_run zeros, then, for every block that is
 *                     not skipped, the levels of each plane with eob[plane]
 *                     != 0 over its in-frame transform blocks (the region
 *                     tile_writer.c:437-456 reads, ending with the last
 *                     transform block's adjusted, at most 32 x 32, area);
 *                     the other planes of such blocks point at the zero run
 *                     (coef_off 0)
 *   frame parameters  the mav1cu_frame_params record of the frame; with
 *                     MAV1CU_EXPORT_LR its lr_type is the one the loop-
 *                     restoration search chose (mav1cu_lr_search)
 *   LR units          (MAV1CU_EXPORT_LR) the frame's mav1cu_lr_unit records,
 *                     all planes (what tile_writer.c's write_lr reads)
 *   reconstruction    (MAV1CU_EXPORT_REC) the shown picture as
 *                     mav1_get_recon returns it (encoder.c:877-915): the
 *                     visible width x height luma samples, then each
 *                     chroma plane's (width+1)/2 x (height+1)/2 samples,
 *                     rows packed
 * Each section starts on a 256-byte boundary at the offset the header gives;
 * the offsets depend on the frame size only. An image's sections read by
 * the reference's writer as its BLOCKS / SBS / COEFS buffers give the same
 * bitstream as the dense buffers. The image never needs more than
 * mav1cu_export_capacity bytes: the level section is at most as long as
 * the dense one. */
typedef struct {
  int32_t status;      /* 0 complete; 1 over capacity; 2 the session's blocks point outside its buffers
                        * (1 and 2: nothing but the header is written) */
  int32_t seq;         /* the session's export count, this export included */
  int32_t num_sbs;     /* superblock table records */
  int32_t num_blocks;  /* mav1cu_block_info records */
  int32_t num_coefs;   /* int32 levels, the zero run included */
  int32_t zero_run;    /* length of the leading run of zero levels */
  int64_t sbs_off;     /* byte offsets of the sections from the start of the image */
  int64_t cdef_off;
  int64_t blocks_off;
  int64_t coefs_off;
  int64_t rec_off;
  int64_t rec_bytes;   /* bytes of the reconstruction section (0 without MAV1CU_EXPORT_REC) */
  int64_t bytes;       /* bytes the export wrote: header and sections */
  int64_t params_off;  /* the frame's mav1cu_frame_params (lr_type as the LR search chose it) */
  int64_t lr_off;      /* lr_units mav1cu_lr_unit records (MAV1CU_EXPORT_LR) */
  int32_t lr_units;
  int32_t pad;
} mav1cu_export_header;

enum { MAV1CU_EXPORT_REC = 1, MAV1CU_EXPORT_LR = 2 };

/* Bytes an export image of this session may need. */
size_t mav1cu_export_capacity(const mav1cu_session *s);
/* The session's own export image (page-locked host memory mapped into the
 * device address space, mav1cu_export_capacity bytes), allocated on the first
 * call and freed with the session; NULL (and a sticky error) if the
 * allocation fails. */
void *mav1cu_export_image(mav1cu_session *s);
/* Enqueues the packing of the current frame's BLOCKS, SBS, COEFS and
 * CDEF_CHOICE (and with MAV1CU_EXPORT_REC in flags its REC) into `image`:
 * page-locked host memory mapped into the device address space
 * (cudaHostAlloc, cudaMallocHost or cudaHostRegister with mapping; the
 * kernels store into it across the bus, so only the packed bytes travel and
 * no copy size is needed up front) or memory of the session's device;
 * 16-byte aligned, at least mav1cu_export_capacity bytes.
 * The packing runs on the session's transfer stream, after the work enqueued
 * on the session's stream so far; the session's next stage that rewrites one
 * of those buffers (analysis, edge types, recon, filter, CDEF selection, an
 * upload or copy) waits for it, and motion search, which does not, overlaps
 * it. The image is complete after mav1cu_synchronize (or, for a stream,
 * mav1cu_stream_synchronize / mav1cu_stream_join, which cover the transfer
 * streams); until then the caller must not read or reuse it. */
int mav1cu_export(mav1cu_session *s, void *image, size_t cap, int flags);
/* Sequence number of the session's last export (the header's seq field);
 * 0 before the first. */
int64_t mav1cu_export_seq(const mav1cu_session *s);
/* Completion of export number seq of the session, for a host consumer that
 * reads images while the device moves on: wait blocks the calling thread
 * (without spinning) until that export's image is complete and returns the
 * session's status (MAV1CU_ERR_DEVICE when a kernel of the session reported
 * an error); query returns 1 when it is complete, 0 when not yet, or a
 * negative status. Any host thread may call them; the thread's current
 * device is set to the session's. The session remembers the last 64
 * exports: for an older seq the wait covers a later export (the transfer
 * stream runs in order). */
int mav1cu_export_wait(mav1cu_session *s, int64_t seq);
int mav1cu_export_query(mav1cu_session *s, int64_t seq);

/* Page-locked host memory, mapped into the address space of every device
 * (cudaHostAlloc, portable and mapped): sources the streams upload
 * asynchronously and export images. NULL on failure. No counterpart in the
 * reference (its buffers are shared with the GPU through unified memory). */
void *mav1cu_host_alloc(size_t bytes);
void mav1cu_host_free(void *p);

/* ---- host helpers (no device work) --------------------------------------- */
/* Forward transform matrices (Q20), 15 x 4096 int32: least-squares inverses
 * of the normative inverse kernels. Replaces fwd_build_matrices
 * (fwd_matrices.c:17-65). */
void mav1cu_build_fwd_matrices(int32_t *mats);

/* ---- edge types without allocation ---------------------------------------- */
/* No counterpart in the reference. The result of mav1cu_edge_types
 * (interp_filter bits 4/5 of every block) on caller-owned device buffers,
 * enqueued on `stream` (a cudaStream_t; NULL is the legacy default stream),
 * without allocating device memory: for hosts that fix their device memory
 * at start-up or whose other streams must not be stalled by cudaMalloc /
 * cudaFree. `params` is a device copy of the frame's mav1cu_frame_params;
 * `blocks` / `sbs` are the analysis output (num_sbs superblocks);
 * mi_rows / mi_cols are the frame's size in 4x4 units and must equal params'
 * mi_rows / mi_cols: blocks at or beyond the given size are left unchanged.
 * Scratch is a fixed device array of 2 x 1,048,576 bytes per device: frames
 * above 1,048,576 4x4 units (4096 x 4096 luma samples) are refused with
 * MAV1CU_ERR_ARG. Each call clears the scratch it uses first. Calls that
 * overlap in time on one device share that scratch and race: order them on
 * one stream or with events. Every call looks up the scratch address on
 * the current device (not cached, so a device reset does not leave a stale
 * address); the first call on a device may load the device code: make it
 * before any stream capture on that device. Returns MAV1CU_OK once the work is enqueued;
 * errors are written to err. */
int mav1cu_edge_types_noalloc(const mav1cu_frame_params *params, mav1cu_block_info *blocks,
                              const mav1cu_sb_info *sbs, int mi_rows, int mi_cols, int num_sbs, void *stream,
                              char *err, size_t errlen);

#ifdef __cplusplus
}
#endif

#endif
