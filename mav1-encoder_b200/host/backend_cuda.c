/*
 * CUDA (B200, sm_100a) backend of the mav1 encoder: the Backend vtable of
 * src/backend.h:10-24 over libmav1cu's C ABI (include/mav1cu.h).
 *
 * This file compiles inside the encoder's source tree (it includes the
 * encoder's backend.h / enc_internal.h) and links libmav1cu.so. Every hook
 * copies its inputs from the encoder's shared buffers (struct Mav1Encoder
 * Bufs, enc_internal.h:81-151) to the device session, runs the device
 * stages on the session's stream, and copies back every output the host
 * steps that follow read, so the driver, tile writer and LR search run
 * unchanged:
 *   motion_search  SRC REF GOLD          -> MVFIELD MVGOLD
 *   analyze        SRC REF GOLD MV*      -> BLOCKS SBS ACOSTS AINFOS
 *   recon          SRC REF GOLD BLOCKS SBS -> REC, writer inputs
 *   frame_core     SRC REF GOLD          -> MV* REC, writer inputs (edge types on the device)
 *   filter         REC LFMASK            -> REC CDEFBUF[0..n)
 *   restore        REC DBK LRUNITS LROUT -> LROUT
 * (the device copies of REC / COEFS are not initialised from the host:
 * recon writes every sample and coefficient the writer and the following
 * stages read). The writer inputs (BLOCKS, SBS, COEFS) come back as the
 * device's compact export (mav1cu_export): only the blocks in use and the
 * levels of coded planes cross the bus, into a page-locked image the
 * session owns, and are copied into the encoder's buffers with first_block
 * and coef_off rewritten, which every host step that follows reads them by
 * (tile_writer.c:449,585, encoder.c:519-574).
 *
 * Selection: backend_cuda_create() is the factory; built with
 * -DMAV1_CUDA_AS_METAL it is also exported as backend_metal_create, so an
 * unchanged encoder.c picks it for cfg.use_metal = 1 (link it instead of
 * backend_metal.m / backend_metal_stub.c).
 *
 * Errors: the stage hooks return void (backend.h); a device error is
 * printed once and is sticky in the session (the next hooks do nothing), as
 * the Metal backend reports command-buffer errors (backend_metal.m:75,383).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "backend.h"
#include "enc_internal.h"
#include "mav1cu.h"

typedef struct {
  Backend base;
  mav1cu_session *s;
  int reported;
} CudaBackend;

static int ok(CudaBackend *cb, int rc) {
  if (rc && !cb->reported) {
    fprintf(stderr, "mav1 cuda backend: %s\n", mav1cu_error_string(cb->s));
    cb->reported = 1;
  }
  return rc == 0;
}

static void put(CudaBackend *cb, int buf, const Buf *b) {
  size_t n = mav1cu_buf_size(cb->s, buf);
  if (b->base && n) ok(cb, mav1cu_upload(cb->s, buf, b->base, n <= b->size ? n : b->size));
}

static void get(CudaBackend *cb, int buf, Buf *b, size_t n) {
  if (b->base && n) ok(cb, mav1cu_download(cb->s, buf, b->base, n <= b->size ? n : b->size));
}

static void frame_inputs(CudaBackend *cb, struct Mav1Encoder *e) {
  ok(cb, mav1cu_set_params(cb->s, (const mav1cu_frame_params *)e->params.base));
  put(cb, MAV1CU_BUF_SRC, &e->src);
  put(cb, MAV1CU_BUF_REF, &e->ref);
  put(cb, MAV1CU_BUF_GOLD, &e->gold);
}

static size_t bsize(CudaBackend *cb, int buf) { return mav1cu_buf_size(cb->s, buf); }

static void export_writer_inputs(CudaBackend *cb) {
  void *img = mav1cu_export_image(cb->s);
  ok(cb, img ? mav1cu_export(cb->s, img, mav1cu_export_capacity(cb->s), 0) : MAV1CU_ERR_NOMEM);
}

static void section(CudaBackend *cb, Buf *dst, const mav1cu_export_header *h, int64_t off, size_t n) {
  if (n > dst->size) {
    ok(cb, MAV1CU_ERR_ARG);
    return;
  }
  memcpy(dst->base, (const char *)h + off, n);
}

/* after the hook's synchronize: the image's sections into the encoder's buffers */
static void unpack_writer_inputs(CudaBackend *cb, struct Mav1Encoder *e) {
  const mav1cu_export_header *h = (const mav1cu_export_header *)mav1cu_export_image(cb->s);
  if (cb->reported || !h) return;
  if (h->status) {
    fprintf(stderr, "mav1 cuda backend: export status %d\n", h->status);
    cb->reported = 1;
    return;
  }
  section(cb, &e->sbs, h, h->sbs_off, (size_t)h->num_sbs * sizeof(mav1cu_sb_info));
  section(cb, &e->blocks, h, h->blocks_off, (size_t)h->num_blocks * sizeof(mav1cu_block_info));
  section(cb, &e->coefs, h, h->coefs_off, (size_t)h->num_coefs * sizeof(int32_t));
}

static void cu_motion_search(Backend *b, struct Mav1Encoder *e) {
  CudaBackend *cb = (CudaBackend *)b;
  frame_inputs(cb, e);
  ok(cb, mav1cu_motion_search(cb->s));
  get(cb, MAV1CU_BUF_MVFIELD, &e->mvfield, bsize(cb, MAV1CU_BUF_MVFIELD));
  get(cb, MAV1CU_BUF_MVGOLD, &e->mvgold, bsize(cb, MAV1CU_BUF_MVGOLD));
  ok(cb, mav1cu_synchronize(cb->s));
}

static void cu_analyze(Backend *b, struct Mav1Encoder *e) {
  CudaBackend *cb = (CudaBackend *)b;
  frame_inputs(cb, e);
  put(cb, MAV1CU_BUF_MVFIELD, &e->mvfield);
  put(cb, MAV1CU_BUF_MVGOLD, &e->mvgold);
  ok(cb, mav1cu_analyze(cb->s));
  get(cb, MAV1CU_BUF_BLOCKS, &e->blocks, bsize(cb, MAV1CU_BUF_BLOCKS));
  get(cb, MAV1CU_BUF_SBS, &e->sbs, bsize(cb, MAV1CU_BUF_SBS));
  get(cb, MAV1CU_BUF_ACOSTS, &e->acosts, bsize(cb, MAV1CU_BUF_ACOSTS));
  get(cb, MAV1CU_BUF_AINFOS, &e->ainfos, bsize(cb, MAV1CU_BUF_AINFOS));
  ok(cb, mav1cu_synchronize(cb->s));
}

static void cu_recon(Backend *b, struct Mav1Encoder *e) {
  CudaBackend *cb = (CudaBackend *)b;
  frame_inputs(cb, e);
  put(cb, MAV1CU_BUF_BLOCKS, &e->blocks); /* edge types may have run on the host */
  put(cb, MAV1CU_BUF_SBS, &e->sbs);
  ok(cb, mav1cu_recon(cb->s));
  get(cb, MAV1CU_BUF_REC, &e->rec, e->frame_bytes);
  export_writer_inputs(cb);
  if (ok(cb, mav1cu_synchronize(cb->s))) unpack_writer_inputs(cb, e);
}

static void cu_frame_core(Backend *b, struct Mav1Encoder *e) {
  CudaBackend *cb = (CudaBackend *)b;
  frame_inputs(cb, e);
  ok(cb, mav1cu_frame_core(cb->s));
  get(cb, MAV1CU_BUF_MVFIELD, &e->mvfield, bsize(cb, MAV1CU_BUF_MVFIELD));
  get(cb, MAV1CU_BUF_MVGOLD, &e->mvgold, bsize(cb, MAV1CU_BUF_MVGOLD));
  get(cb, MAV1CU_BUF_REC, &e->rec, e->frame_bytes);
  export_writer_inputs(cb);
  if (ok(cb, mav1cu_synchronize(cb->s))) unpack_writer_inputs(cb, e);
}

static void cu_filter(Backend *b, struct Mav1Encoder *e) {
  CudaBackend *cb = (CudaBackend *)b;
  int n = e->num_cdef_presets;
  ok(cb, mav1cu_set_params(cb->s, (const mav1cu_frame_params *)e->params.base));
  put(cb, MAV1CU_BUF_REC, &e->rec);
  put(cb, MAV1CU_BUF_LFMASK, &e->lfmask);
  ok(cb, mav1cu_filter(cb->s, n));
  get(cb, MAV1CU_BUF_REC, &e->rec, e->frame_bytes);
  if (n) get(cb, MAV1CU_BUF_CDEFBUF, &e->cdefbuf, (size_t)n * e->frame_bytes);
  ok(cb, mav1cu_synchronize(cb->s));
}

static void cu_restore(Backend *b, struct Mav1Encoder *e) {
  CudaBackend *cb = (CudaBackend *)b;
  ok(cb, mav1cu_set_params(cb->s, (const mav1cu_frame_params *)e->params.base));
  put(cb, MAV1CU_BUF_REC, &e->rec);
  put(cb, MAV1CU_BUF_DBK, &e->dbk);
  put(cb, MAV1CU_BUF_LRUNITS, &e->lrunits);
  put(cb, MAV1CU_BUF_LROUT, &e->lrout);
  ok(cb, mav1cu_restore(cb->s));
  get(cb, MAV1CU_BUF_LROUT, &e->lrout, e->frame_bytes);
  ok(cb, mav1cu_synchronize(cb->s));
}

static void cu_destroy(Backend *b) {
  CudaBackend *cb = (CudaBackend *)b;
  mav1cu_session_destroy(cb->s);
  free(cb);
}

Backend *backend_cuda_create(struct Mav1Encoder *e, char *err, size_t errlen) {
  mav1cu_session *s = NULL;
  if (mav1cu_session_create(e->w, e->h, 4, &s, err, errlen) != MAV1CU_OK) return NULL;
  CudaBackend *cb = calloc(1, sizeof(*cb));
  cb->s = s;
  cb->base.name = "cuda";
  cb->base.motion_search = cu_motion_search;
  cb->base.analyze = cu_analyze;
  cb->base.recon = cu_recon;
  cb->base.filter = cu_filter;
  cb->base.restore = cu_restore;
  cb->base.destroy = cu_destroy;
  cb->base.frame_core = cu_frame_core;
  /* the encoder's forward matrices (the session derives the same table) */
  ok(cb, mav1cu_upload(s, MAV1CU_BUF_MATS, e->mats.base, mav1cu_buf_size(s, MAV1CU_BUF_MATS)));
  return &cb->base;
}

#ifdef MAV1_CUDA_AS_METAL
Backend *backend_metal_create(struct Mav1Encoder *e, char *err, size_t errlen) {
  return backend_cuda_create(e, err, errlen);
}
#endif
