/* ORACLE — test infrastructure only; never linked into the product.
 *
 * The reference's frame driver (src/encoder.c) restated for Linux without
 * Apple libdispatch / clang Blocks, in the reference's own serial mode
 * (MAV1_NOASYNC: no frame engines, no writer queue, every job inline;
 * encoder.c:124,1168-1224 take that path when the queues are absent). The
 * reference's comments state that the serial and concurrent modes emit the
 * same bytes. Everything else it calls is the reference's own code compiled
 * in place: kernels (src/kernels/k_*.h), tile writer, OBU writer, entropy
 * coder, motion-vector prediction, LR search and forward matrices.
 *
 * Additions for the tests, none of which changes an output byte:
 *  - oref_set_hook: a callback after each stage of run_frame_core, so a test
 *    can snapshot the backend's inputs and outputs per frame;
 *  - oref_set_backend_factory: the function create_enc calls when
 *    cfg.use_metal is set (default: the reference's Metal stub, which fails),
 *    so the CUDA backend can be driven through the unchanged vtable;
 *  - oref_buf / oref_geometry: raw access to the encoder's buffers.
 */
#include <math.h>
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "backend.h"
#include "enc_internal.h"
#include "fwd_matrices.h"
#include "kernels/k_analysis.h"
#include "kernels/k_fwd.h"
#include "kernels/k_lr.h"
#include "kernels/k_me.h"
#include "kernels/k_recon.h"

/* ---- test hooks ---------------------------------------------------------- */

enum {
  OREF_STAGE_PARAMS = 0,   /* setup_params done; src / ref / gold loaded */
  OREF_STAGE_ME = 1,       /* be->motion_search */
  OREF_STAGE_ANALYZE = 2,  /* be->analyze */
  OREF_STAGE_EDGE = 3,     /* edge_filter_types */
  OREF_STAGE_RECON = 4,    /* be->recon */
  OREF_STAGE_FINFO = 5,    /* build_filter_info */
  OREF_STAGE_FILTER = 6,   /* be->filter */
  OREF_STAGE_CDEFSEL = 7,  /* cdef_select */
  OREF_STAGE_LRSEL = 8,    /* lr_select */
  OREF_STAGE_RESTORE = 9,  /* be->restore (before the rec / lrout swap) */
  OREF_STAGE_DONE = 10,    /* run_frame_core finished */
};

typedef void (*oref_hook_fn)(void *user, int stage, struct Mav1Encoder *e);
static oref_hook_fn g_hook;
static void *g_hook_user;
void oref_set_hook(oref_hook_fn fn, void *user) {
  g_hook = fn;
  g_hook_user = user;
}
#define HOOK(st, e) \
  do { \
    if (g_hook) g_hook(g_hook_user, (st), (e)); \
  } while (0)

typedef Backend *(*oref_factory_fn)(struct Mav1Encoder *e, char *err, size_t errlen);
static oref_factory_fn g_factory;
void oref_set_backend_factory(oref_factory_fn fn) { g_factory = fn; }

/* ---- buffers ------------------------------------------------------------- */

#define PAGE 16384

static double now(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + ts.tv_nsec * 1e-9;
}

/* encoder.c:30-39: zero-filled, page-rounded allocation */
static int buf_alloc(Buf *b, size_t size) {
  size = (size + PAGE - 1) / PAGE * PAGE;
  if (size == 0) size = PAGE;
  void *p = NULL;
  if (posix_memalign(&p, 4096, size)) return -1;
  memset(p, 0, size);
  b->base = p;
  b->size = size;
  return 0;
}

static void buf_free(Buf *b) {
  free(b->base);
  b->base = NULL;
}

static int env_or(const char *n, int d) {
  const char *v = getenv(n);
  return v ? atoi(v) : d;
}

/* encoder.c:51-66 */
void mav1_default_config(Mav1Config *cfg, int width, int height) {
  memset(cfg, 0, sizeof(*cfg));
  cfg->width = width;
  cfg->height = height;
  cfg->qindex = 100;
  cfg->use_metal = 1;
  cfg->keyint = 0;
  cfg->tx_search = 1;
  cfg->tx_depth = 1;
  cfg->restoration = 1;
  cfg->switchable_interp = 1;
  cfg->intra_edge_filter = 1;
  cfg->loop_filter = 1;
  cfg->cdef = 1;
  cfg->me_range = 32;
}

/* encoder.c:69-226, serial mode (no driver / engine split, no writer queue) */
Mav1Encoder *mav1_create(const Mav1Config *cfg, char *err, size_t errlen) {
  if (cfg->width < 16 || cfg->height < 16 || cfg->width > 65536 || cfg->height > 65536) {
    snprintf(err, errlen, "unsupported frame size %dx%d", cfg->width, cfg->height);
    return NULL;
  }
  Mav1Encoder *e = calloc(1, sizeof(*e));
  e->cfg = *cfg;
  if (e->cfg.turbo) {
    e->cfg.fast = 1;
    if (e->cfg.altref < 2) e->cfg.altref = 2;
    e->cfg.leaf = 1;
  }
  if (e->cfg.altref == 1) e->cfg.altref = 0;
  if (e->cfg.altref > 16) e->cfg.altref = 16;
  if (e->cfg.altref) e->cfg.multi_ref = e->cfg.nonref_odd = 0;
  if (!e->cfg.altref) e->cfg.leaf = 0;
  e->leafopt_cfg = getenv("MAV1_LEAFOPT") ? (int)strtol(getenv("MAV1_LEAFOPT"), NULL, 0) : 0x3F;
  if (e->cfg.qindex < 0) e->cfg.qindex = 0;
  if (e->cfg.qindex > 255) e->cfg.qindex = 255;
  e->w = cfg->width;
  e->h = cfg->height;
  e->mi_cols = 2 * ((e->w + 7) >> 3);
  e->mi_rows = 2 * ((e->h + 7) >> 3);
  e->sb_cols = (e->mi_cols + 15) >> 4;
  e->sb_rows = (e->mi_rows + 15) >> 4;
  e->num_sbs = e->sb_cols * e->sb_rows;
  {
    int k = 0;
    while (((MAX_TILE_WIDTH >> 6) << k) < e->sb_cols) k++;
    e->min_log2_tile_cols = k;
    int maxCols = e->sb_cols < MAX_TILE_COLS ? e->sb_cols : MAX_TILE_COLS;
    for (k = 0; (1 << k) < maxCols; k++) {
    }
    e->max_log2_tile_cols = k;
    int l = e->cfg.tile_cols_log2;
    if (l < e->min_log2_tile_cols) l = e->min_log2_tile_cols;
    if (l > e->max_log2_tile_cols) l = e->max_log2_tile_cols;
    e->tile_cols_log2 = l;
    e->tile_w_sb = (e->sb_cols + (1 << l) - 1) >> l;
    e->tile_cols = (e->sb_cols + e->tile_w_sb - 1) / e->tile_w_sb;
  }
  e->stride[0] = e->sb_cols * 64;
  e->stride[1] = e->stride[2] = e->sb_cols * 32;
  e->plane_h[0] = e->sb_rows * 64;
  e->plane_h[1] = e->plane_h[2] = e->sb_rows * 32;
  e->offset[0] = 0;
  e->offset[1] = e->stride[0] * e->plane_h[0];
  e->offset[2] = e->offset[1] + e->stride[1] * e->plane_h[1];
  e->frame_bytes = (size_t)e->offset[2] + (size_t)e->stride[2] * e->plane_h[2];

  int ok = 0;
  ok |= buf_alloc(&e->src, e->frame_bytes);
  ok |= buf_alloc(&e->rec, e->frame_bytes);
  ok |= buf_alloc(&e->ref, e->frame_bytes);
  int ref2 = e->cfg.multi_ref || e->cfg.altref;
  if (ref2) ok |= buf_alloc(&e->gold, e->frame_bytes);
  if (e->cfg.altref) {
    ok |= buf_alloc(&e->slot[0], e->frame_bytes);
    ok |= buf_alloc(&e->slot[2], e->frame_bytes);
    ok |= buf_alloc(&e->slot[3], e->frame_bytes);
    if (e->cfg.leaf)
      for (int i = 4; i < 8; i++) ok |= buf_alloc(&e->slot[i], e->frame_bytes);
    e->inq = calloc((size_t)e->cfg.altref + 1, sizeof *e->inq);
  }
  ok |= buf_alloc(&e->params, sizeof(FrameParams));
  ok |= buf_alloc(&e->blocks, sizeof(BlockInfo) * MAX_BLOCKS_PER_SB * e->num_sbs);
  ok |= buf_alloc(&e->sbs, sizeof(SbInfo) * e->num_sbs);
  ok |= buf_alloc(&e->coefs, sizeof(int32_t) * COEFS_PER_SB * e->num_sbs);
  ok |= buf_alloc(&e->mats, sizeof(int32_t) * FWD_SLOT_SIZE * FWD_NUM_SLOTS);
  ok |= buf_alloc(&e->mvfield, sizeof(int32_t) * 2 * NUM_NODES * e->num_sbs);
  ok |= buf_alloc(&e->mvgold, ref2 ? sizeof(int32_t) * 2 * NUM_NODES * e->num_sbs : 0);
  ok |= buf_alloc(&e->acosts, sizeof(long) * A_ITEMS * (size_t)e->num_sbs);
  ok |= buf_alloc(&e->ainfos, sizeof(BlockInfo) * A_ITEMS * (size_t)e->num_sbs);
  ok |= buf_alloc(&e->hpel, e->cfg.turbo ? (size_t)(ME_QP_ENTRIES * 16 + 1) * e->w * e->h +
                                               (size_t)(ME_QP_ENTRIES + 1) * ((e->w + 3) >> 2) * ((e->h + 3) >> 2)
                                         : 0);
  ok |= buf_alloc(&e->scratch, sizeof(int32_t) * SCRATCH_INTS * (size_t)e->num_sbs);
  ok |= buf_alloc(&e->lfmask, (size_t)e->mi_rows * e->mi_cols);
  ok |= buf_alloc(&e->dbk, e->frame_bytes);
  ok |= buf_alloc(&e->lrout, e->frame_bytes);
  ok |= buf_alloc(&e->lrunits, sizeof(LrUnit) * 3 * (size_t)(e->sb_rows + 1) * (e->sb_cols + 1));
  e->num_cdef_presets = e->cfg.cdef ? 4 : 0;
  ok |= buf_alloc(&e->cdefbuf, e->frame_bytes * (e->num_cdef_presets ? e->num_cdef_presets : 1));
  if (ok) {
    snprintf(err, errlen, "out of memory");
    mav1_destroy(e);
    return NULL;
  }
  fwd_build_matrices((int32_t *)e->mats.base);
  e->mi = calloc((size_t)e->mi_rows * e->mi_cols, sizeof(MiInfo));
  e->cdef_idx = calloc((size_t)e->num_sbs, 1);
  e->cdef_choice = calloc((size_t)e->num_sbs, 1);
  if (cfg->use_metal) {
    e->be = g_factory ? g_factory(e, err, errlen) : backend_metal_create(e, err, errlen);
    if (!e->be) {
      mav1_destroy(e);
      return NULL;
    }
  } else {
    e->be = backend_cpu_create(e);
  }
  return e;
}

/* encoder.c:230-288 */
void mav1_destroy(Mav1Encoder *e) {
  if (!e) return;
  if (e->be) e->be->destroy(e->be);
  buf_free(&e->src);
  buf_free(&e->rec);
  buf_free(&e->ref);
  buf_free(&e->gold);
  for (int i = 0; i < 8; i++) buf_free(&e->slot[i]);
  for (int i = 0; i < e->inq_n; i++) free(e->inq[i]);
  free(e->inq);
  for (int i = e->out_pos; i < e->out_n; i++) {
    free(e->outq[i].data);
    free(e->outq[i].recon);
  }
  free(e->outq);
  free(e->shown_recon);
  if (e->pending) free(e->pend_data);
  buf_free(&e->mvgold);
  buf_free(&e->params);
  buf_free(&e->blocks);
  buf_free(&e->sbs);
  buf_free(&e->coefs);
  buf_free(&e->mats);
  buf_free(&e->mvfield);
  buf_free(&e->scratch);
  buf_free(&e->hpel);
  buf_free(&e->acosts);
  buf_free(&e->ainfos);
  free(e->mi);
  free(e->cdef_idx);
  free(e->cdef_choice);
  buf_free(&e->lfmask);
  buf_free(&e->cdefbuf);
  buf_free(&e->dbk);
  buf_free(&e->lrout);
  buf_free(&e->lrunits);
  free(e);
}

const char *mav1_backend_name(const Mav1Encoder *e) { return e->be->name; }
const Mav1FrameStats *mav1_last_stats(const Mav1Encoder *e) { return &e->last; }
size_t mav1_sequence_header(const Mav1Encoder *e, uint8_t *out) { return write_sequence_header(e, out); }

/* encoder.c:297-310 */
static void load_source(Mav1Encoder *e, const uint8_t *const planes[3], const int strides[3]) {
  for (int p = 0; p < 3; p++) {
    int pw = p ? (e->w + 1) >> 1 : e->w;
    int ph = p ? (e->h + 1) >> 1 : e->h;
    int aw = e->stride[p], ah = e->plane_h[p];
    uint8_t *dst = e->src.base + e->offset[p];
    for (int y = 0; y < ah; y++) {
      const uint8_t *s = planes[p] + (size_t)(y < ph ? y : ph - 1) * strides[p];
      uint8_t *d = dst + (size_t)y * aw;
      memcpy(d, s, pw);
      memset(d + pw, s[pw - 1], aw - pw);
    }
  }
}

/* encoder.c:315-346 */
static int smooth_mode(int m) { return m == SMOOTH_PRED || m == SMOOTH_V_PRED || m == SMOOTH_H_PRED; }

void edge_types_rows(Mav1Encoder *e, uint8_t *ys, uint8_t *uvs, int row0, int row1) {
  const FrameParams *fp = ENC_PARAMS(e);
  int cols = e->mi_cols, rows = e->mi_rows;
  BlockInfo *blocks = ENC_BLOCKS(e);
  const SbInfo *sbs = ENC_SBS(e);
  int s0 = row0 * e->sb_cols, s1 = row1 * e->sb_cols;
  for (int s = s0; s < s1; s++)
    for (int i = 0; i < sbs[s].num_blocks; i++) {
      const BlockInfo *b = &blocks[sbs[s].first_block + i];
      int ysm = smooth_mode(b->y_mode) && !b->is_inter, uvsm = !b->is_inter && smooth_mode(b->uv_mode);
      for (int r = b->mi_row; r < b->mi_row + Num_4x4_Blocks_High[b->bsize] && r < rows; r++)
        for (int c = b->mi_col; c < b->mi_col + Num_4x4_Blocks_Wide[b->bsize] && c < cols; c++) {
          ys[r * cols + c] = (uint8_t)ysm;
          uvs[r * cols + c] = (uint8_t)uvsm;
        }
    }
  for (int s = s0; s < s1; s++)
    for (int i = 0; i < sbs[s].num_blocks; i++) {
      BlockInfo *b = &blocks[sbs[s].first_block + i];
      int r = b->mi_row, c = b->mi_col;
      int availU = r > 0, availL = c > tile_col_start(fp, c);
      int fy = (availU && ys[(r - 1) * cols + c]) || (availL && ys[r * cols + c - 1]);
      int fuv = (availU && uvs[(r - 1) * cols + k_min(c + 1, cols - 1)]) ||
                (availL && uvs[k_min(r + 1, rows - 1) * cols + c - 1]);
      b->interp_filter = (b->interp_filter & 15) | fy << 4 | fuv << 5;
    }
}

/* encoder.c:399-404 */
static void edge_filter_types(Mav1Encoder *e) {
  uint8_t *ys = calloc((size_t)e->mi_rows * e->mi_cols, 1), *uvs = calloc((size_t)e->mi_rows * e->mi_cols, 1);
  edge_types_rows(e, ys, uvs, 0, e->sb_rows);
  free(ys);
  free(uvs);
}

/* encoder.c:407-510 */
static void setup_params(Mav1Encoder *e, int isKey) {
  FrameParams *fp = ENC_PARAMS(e);
  memset(fp, 0, sizeof(*fp));
  fp->mi_cols = e->mi_cols;
  fp->mi_rows = e->mi_rows;
  fp->sb_cols = e->sb_cols;
  fp->sb_rows = e->sb_rows;
  for (int p = 0; p < 3; p++) {
    fp->plane_w[p] = e->stride[p];
    fp->plane_h[p] = e->plane_h[p];
    fp->stride[p] = e->stride[p];
    fp->offset[p] = e->offset[p];
  }
  int q = e->hdr.base_q_idx;
  fp->base_q_idx = q;
  for (int p = 0; p < 3; p++) {
    fp->dc_q[p] = Dc_Qlookup[0][q];
    fp->ac_q[p] = Ac_Qlookup[0][q];
  }
  fp->frame_is_intra = isKey;
  fp->reduced_tx_set = 0;
  fp->enable_intra_edge_filter = e->cfg.intra_edge_filter;
  fp->tx_search = e->cfg.tx_search;
  fp->lossless = q == 0;
  fp->tx_mode_select = q != 0 && e->cfg.tx_depth;
  fp->switchable_interp = !isKey && e->cfg.switchable_interp;
  fp->golden = !isKey && e->cfg.multi_ref && e->gold_id != e->last_id;
  fp->ref2_frame = GOLDEN_FRAME;
  if (e->cfg.altref) {
    fp->golden = !isKey && e->frame_kind >= 2;
    fp->ref2_frame = ALTREF_FRAME;
    fp->compound = e->hdr.reference_select;
  }
  fp->fast = e->cfg.fast;
  fp->turbo = e->cfg.turbo ? (getenv("MAV1_TURBO") ? (int)strtol(getenv("MAV1_TURBO"), NULL, 0) : 0x47CBF1) : 0;
  fp->leaf = e->cfg.leaf ? (e->leafopt & 1) : e->nonref && !getenv("MAV1_LEAFINTRA");
  if (e->leafopt & 16) fp->tx_search = 0;
  {
    int dt = getenv("MAV1_DT") ? atoi(getenv("MAV1_DT")) : e->sb_rows >= 16 ? 320 : 352;
    int bias = getenv("MAV1_DTB") ? atoi(getenv("MAV1_DTB")) : 0;
    fp->depth_thr = e->cfg.turbo ? dt * (q + bias) / (128 + bias) : 0;
  }
  fp->tile_w_sb = e->tile_w_sb;
  long acq = fp->ac_q[0];
  fp->lambda = (int32_t)(acq * acq * 256 / 430);
  fp->frame_w = e->w;
  fp->frame_h = e->h;
  fp->me_range = e->cfg.me_range;
  if ((e->leafopt & 32) && fp->me_range > 16) fp->me_range = 16;

  FrameHdr *h = &e->hdr;
  int lvl = 0;
  if (e->cfg.loop_filter && q > 0 && !(e->cfg.leaf ? (e->leafopt & 2) : e->nonref && !getenv("MAV1_LEAFLF"))) {
    lvl = (int)((acq * 20723 + 1015158 + (1 << 17)) >> 18);
    if (!isKey) lvl -= 4;
    lvl = lvl < 0 ? 0 : (lvl > MAX_LOOP_FILTER ? MAX_LOOP_FILTER : lvl);
  }
  for (int i = 0; i < 4; i++) h->lf_level[i] = fp->lf_level[i] = lvl;
  h->lf_sharpness = fp->lf_sharpness = 0;
  static const int presets[4][4] = {{0, 0, 0, 0}, {2, 1, 1, 0}, {4, 2, 2, 1}, {8, 4, 4, 2}};
  h->cdef_damping = fp->cdef_damping = 3 + (q >> 6);
  h->cdef_bits = fp->cdef_bits = 2;
  if (e->leafopt & 4) {
    h->cdef_damping = fp->cdef_damping = 3;
    h->cdef_bits = fp->cdef_bits = 0;
  }
  int pi[4] = {0, 1, 2, 3};
  if ((fp->turbo & 2048) && h->cdef_bits == 2) {
    h->cdef_bits = fp->cdef_bits = 1;
    pi[1] = env_or("MAV1_CP", 2);
  }
  for (int i = 0; i < 4; i++) {
    const int *ps = presets[pi[i]];
    h->cdef_y_pri[i] = fp->cdef_y_pri[i] = ps[0];
    h->cdef_y_sec[i] = fp->cdef_y_sec[i] = ps[1];
    h->cdef_uv_pri[i] = fp->cdef_uv_pri[i] = ps[2];
    h->cdef_uv_sec[i] = fp->cdef_uv_sec[i] = ps[3];
  }
  int off = 0;
  for (int p = 0; p < 3; p++) {
    int sub = p > 0, size = RESTORATION_TILESIZE_MAX >> 2;
    int pw = (e->w + sub) >> sub, ph = (e->h + sub) >> sub;
    fp->lr_type[p] = h->lr_type[p] = RESTORE_NONE;
    fp->lr_unit_size[p] = size;
    fp->lr_unit_rows[p] = k_max((ph + (size >> 1)) / size, 1);
    fp->lr_unit_cols[p] = k_max((pw + (size >> 1)) / size, 1);
    fp->lr_unit_off[p] = off;
    off += fp->lr_unit_rows[p] * fp->lr_unit_cols[p];
  }
}

/* encoder.c:513-526 */
static void build_filter_info(Mav1Encoder *e) {
  uint8_t *info = e->lfmask.base;
  const SbInfo *sbs = ENC_SBS(e);
  const BlockInfo *blocks = ENC_BLOCKS(e);
  for (int i = 0; i < e->num_sbs; i++)
    for (int k = 0; k < sbs[i].num_blocks; k++) {
      const BlockInfo *b = &blocks[sbs[i].first_block + k];
      int skip = b->eob[0] == 0 && b->eob[1] == 0 && b->eob[2] == 0;
      int bw4 = Num_4x4_Blocks_Wide[b->bsize], bh4 = Num_4x4_Blocks_High[b->bsize];
      for (int y = 0; y < bh4 && b->mi_row + y < e->mi_rows; y++)
        for (int x = 0; x < bw4 && b->mi_col + x < e->mi_cols; x++)
          info[(b->mi_row + y) * e->mi_cols + b->mi_col + x] = (uint8_t)(b->bsize | (skip << 5) | (b->tx_depth << 6));
    }
}

/* encoder.c:530-563 (the dispatch_apply over superblocks as an OpenMP loop) */
static void cdef_select(Mav1Encoder *e) {
#pragma omp parallel for schedule(dynamic, 4)
  for (int sb = 0; sb < e->num_sbs; sb++) {
    int sr = sb / e->sb_cols, sc = sb % e->sb_cols;
    long best = -1;
    int bestK = 0;
    for (int k = 0; k < e->num_cdef_presets; k++) {
      const uint8_t *out = e->cdefbuf.base + (size_t)k * e->frame_bytes;
      long sse = 0;
      for (int p = 0; p < 3; p++) {
        int sub = p > 0, n = 64 >> sub;
        int pw = p ? (e->w + 1) >> 1 : e->w, ph = p ? (e->h + 1) >> 1 : e->h;
        for (int y = sr * n; y < (sr + 1) * n && y < ph; y++)
          for (int x = sc * n; x < (sc + 1) * n && x < pw; x++) {
            size_t o = e->offset[p] + (size_t)y * e->stride[p] + x;
            int d = (int)out[o] - (int)e->src.base[o];
            sse += d * d;
          }
      }
      if (best < 0 || sse < best) {
        best = sse;
        bestK = k;
      }
    }
    e->cdef_choice[sb] = (int8_t)bestK;
    const uint8_t *out = e->cdefbuf.base + (size_t)bestK * e->frame_bytes;
    for (int p = 0; p < 3; p++) {
      int sub = p > 0, n = 64 >> sub;
      int mw = (e->mi_cols * 4) >> sub, mh = (e->mi_rows * 4) >> sub;
      for (int y = sr * n; y < (sr + 1) * n && y < mh; y++) {
        int x0 = sc * n, x1 = (sc + 1) * n < mw ? (sc + 1) * n : mw;
        size_t o = e->offset[p] + (size_t)y * e->stride[p];
        memcpy(e->rec.base + o + x0, out + o + x0, x1 - x0);
      }
    }
  }
}

/* encoder.c:565-579 */
const char *const mav1_tool_names[16] = {"intra", "inter", "cfl", "angle_delta", "tx_non_dct", "skip",
                                          "rect_part", "compound", "obmc", "lr_wiener_units", "lr_sgr_units",
                                          "golden", "altref", "", "", ""};

static void count_tools(Mav1FrameStats *st, const BlockInfo *b) {
  st->tool_use[0] += !b->is_inter;
  st->tool_use[1] += b->is_inter;
  st->tool_use[2] += !b->is_inter && b->uv_mode == UV_CFL_PRED;
  st->tool_use[3] += !b->is_inter && (b->angle_y != 0 || b->angle_uv != 0);
  st->tool_use[4] += b->eob[0] > 0 && b->tx_type != DCT_DCT;
  st->tool_use[5] += b->eob[0] == 0 && b->eob[1] == 0 && b->eob[2] == 0;
  st->tool_use[6] += Block_Width(b->bsize) != Block_Height(b->bsize);
  st->tool_use[7] += b->is_inter && b->ref_frame1 > INTRA_FRAME;
  st->tool_use[11] += b->is_inter && b->ref_frame == GOLDEN_FRAME;
  st->tool_use[12] += b->is_inter && b->ref_frame == ALTREF_FRAME;
}

/* encoder.c:585-595 */
static int frame_qindex(const Mav1Encoder *e, int isKey) {
  int q = e->cfg.qindex;
  if (q == 0) return 0;
  int off = isKey ? env_or("MAV1_QK", -24) : (e->order_hint % 4 == 0 ? env_or("MAV1_Q4", -8) : env_or("MAV1_QP", 4));
  if (!isKey && e->nonref) off = env_or("MAV1_QN", 12);
  if (!isKey && e->cfg.altref) off = e->frame_kind == 1 ? env_or("MAV1_QA", -8) : env_or("MAV1_QP", 4);
  if (!isKey && e->cfg.leaf && e->frame_kind == 3) off = env_or("MAV1_QM", 0);
  if (!isKey && e->cfg.leaf && e->nonref) off = env_or("MAV1_QL", 8);
  q += off;
  return q < 1 ? 1 : q > 255 ? 255 : q;
}

/* encoder.c:599-657 (the Metal frame_core branch is taken by any backend
 * that provides one, exactly as the reference does) */
static void run_frame_core(Mav1Encoder *e, int isKey) {
  setup_params(e, isKey);
  HOOK(OREF_STAGE_PARAMS, e);
  double t0 = now(), t1, t2;
  if (e->cfg.turbo && e->be->frame_core) {
    e->be->frame_core(e->be, e);
    t1 = t0;
    t2 = now();
    HOOK(OREF_STAGE_RECON, e);
  } else {
    if (!isKey) e->be->motion_search(e->be, e);
    HOOK(OREF_STAGE_ME, e);
    e->be->analyze(e->be, e);
    HOOK(OREF_STAGE_ANALYZE, e);
    if (e->cfg.intra_edge_filter) edge_filter_types(e);
    HOOK(OREF_STAGE_EDGE, e);
    t1 = now();
    e->be->recon(e->be, e);
    t2 = now();
    HOOK(OREF_STAGE_RECON, e);
  }
  int cdefOff = (e->leafopt & 4) != 0, nPresets = e->num_cdef_presets;
  int lfOn = e->hdr.lf_level[0] || e->hdr.lf_level[1] || e->hdr.lf_level[2] || e->hdr.lf_level[3];
  int filt = lfOn || (nPresets && !cdefOff) || !e->cfg.turbo;
  if (filt) build_filter_info(e);
  HOOK(OREF_STAGE_FINFO, e);
  if (nPresets) e->num_cdef_presets = 1 << e->hdr.cdef_bits;
  if (cdefOff) {
    e->num_cdef_presets = 0;
    memset(e->cdef_choice, 0, (size_t)e->num_sbs);
  }
  if (filt) e->be->filter(e->be, e);
  HOOK(OREF_STAGE_FILTER, e);
  e->num_cdef_presets = nPresets;
  int useLr = e->cfg.restoration && e->cfg.qindex > 0 && !(e->leafopt & 8);
  if (useLr) memcpy(e->dbk.base, e->rec.base, e->frame_bytes);
  if (e->cfg.cdef && e->cfg.qindex > 0 && !cdefOff) cdef_select(e);
  HOOK(OREF_STAGE_CDEFSEL, e);
  if (useLr) {
    lr_select(e);
    HOOK(OREF_STAGE_LRSEL, e);
    memcpy(e->lrout.base, e->rec.base, e->frame_bytes);
    e->be->restore(e->be, e);
    HOOK(OREF_STAGE_RESTORE, e);
    Buf t = e->rec;
    e->rec = e->lrout;
    e->lrout = t;
  }
  double t3 = now();
  e->last.t_analysis = t1 - t0;
  e->last.t_recon = t2 - t1;
  e->last.t_filter = t3 - t2;
  e->last.t_entropy = 0;
  HOOK(OREF_STAGE_DONE, e);
}

/* encoder.c:659-704 (MAV1_DUMP_DEC decision dump) */
static void dump_decisions(Mav1Encoder *s, size_t tileSize) {
  static pthread_mutex_t mu = PTHREAD_MUTEX_INITIALIZER;
  static FILE *f;
  static char fpath[1024];
  const char *path = getenv("MAV1_DUMP_DEC");
  if (!path) return;
  int rows8 = (s->mi_rows + 1) >> 1, cols8 = (s->mi_cols + 1) >> 1;
  size_t cells = (size_t)rows8 * cols8;
  uint8_t *grid = calloc(cells, 8);
  const SbInfo *sbs = ENC_SBS(s);
  const BlockInfo *blocks = ENC_BLOCKS(s);
  for (int i = 0; i < s->num_sbs; i++)
    for (int k = 0; k < sbs[i].num_blocks; k++) {
      const BlockInfo *b = &blocks[sbs[i].first_block + k];
      int w8 = (Num_4x4_Blocks_Wide[b->bsize] + 1) >> 1, h8 = (Num_4x4_Blocks_High[b->bsize] + 1) >> 1;
      int r0 = b->mi_row >> 1, c0 = b->mi_col >> 1;
      for (int r = r0; r < r0 + h8 && r < rows8; r++)
        for (int c = c0; c < c0 + w8 && c < cols8; c++) {
          uint8_t *cell = grid + ((size_t)r * cols8 + c) * 8;
          cell[0] = (uint8_t)b->bsize;
          cell[1] = !b->is_inter ? 0 : b->ref_frame1 ? 2 : 1;
          cell[2] = (uint8_t)b->ref_frame;
          cell[3] = 0;
          int16_t mr = (int16_t)b->mv_row, mc = (int16_t)b->mv_col;
          memcpy(cell + 4, &mr, 2);
          memcpy(cell + 6, &mc, 2);
        }
    }
  int32_t hdr[11] = {0x4345444D, s->order_hint, s->dump_last_hint, s->dump_arf_hint,
                     s->hdr.frame_type == KEY_FRAME ? 0 : 1, s->frame_kind, s->nonref, s->hdr.base_q_idx,
                     rows8, cols8, (int32_t)tileSize};
  pthread_mutex_lock(&mu);
  /* a new path (a later encode in the same process) starts a new file */
  if (f && strcmp(fpath, path)) {
    fclose(f);
    f = NULL;
  }
  if (!f) {
    f = fopen(path, "wb");
    snprintf(fpath, sizeof fpath, "%s", path);
  }
  if (f) {
    fwrite(hdr, sizeof hdr, 1, f);
    fwrite(grid, 8, cells, f);
    fflush(f);
  }
  pthread_mutex_unlock(&mu);
  free(grid);
}

/* encoder.c:708-725 */
static size_t frame_tail(Mav1Encoder *s, uint8_t **tile, Mav1FrameStats *st) {
  double t3 = now();
  size_t tileSize = write_tile(s, tile);
  dump_decisions(s, tileSize);
  const SbInfo *sbs = ENC_SBS(s);
  const BlockInfo *blocks = ENC_BLOCKS(s);
  for (int i = 0; i < s->num_sbs; i++) {
    st->num_blocks += sbs[i].num_blocks;
    for (int k = 0; k < sbs[i].num_blocks; k++) {
      const BlockInfo *b = &blocks[sbs[i].first_block + k];
      st->num_inter_blocks += b->is_inter;
      count_tools(st, b);
    }
  }
  st->t_entropy += now() - t3;
  return tileSize;
}

/* encoder.c:822-875 */
int mav1_encode(Mav1Encoder *e, const uint8_t *const planes[3], const int strides[3], uint8_t **out,
                size_t *outSize) {
  int isKey = e->frame_num == 0 || (e->cfg.keyint > 0 && e->frame_num % e->cfg.keyint == 0);
  memset(&e->last, 0, sizeof(e->last));
  e->last.frame_type = isKey ? 0 : 1;
  load_source(e, planes, strides);
  FrameHdr *h = &e->hdr;
  memset(h, 0, sizeof(*h));
  e->nonref = !isKey && e->cfg.nonref_odd && (e->order_hint & 1);
  h->frame_type = isKey ? KEY_FRAME : INTER_FRAME;
  h->base_q_idx = frame_qindex(e, isKey);
  if (isKey) e->order_hint = 0;
  h->order_hint = e->order_hint;
  h->show_frame = 1;
  e->dump_last_hint = isKey ? -1 : e->order_hint - 1 - (e->cfg.nonref_odd && (e->order_hint & 1) == 0 ? 1 : 0);
  e->dump_arf_hint = -1;
  if (e->cfg.multi_ref) h->ref_idx[GOLDEN_FRAME - LAST_FRAME] = 1;
  e->golden_refresh = !isKey && !e->nonref && e->cfg.multi_ref && e->order_hint % 4 == 0;
  h->refresh_frame_flags = isKey ? 0xFF : (e->nonref ? 0x00 : 0x01 | (e->golden_refresh ? 0x02 : 0));

  uint8_t *tile = NULL;
  run_frame_core(e, isKey);
  size_t tileSize = frame_tail(e, &tile, &e->last);
  double t3 = now();
  size_t cap = tileSize + 1024;
  uint8_t *buf = malloc(cap);
  size_t pos = write_temporal_delimiter(buf);
  if (isKey) pos += write_sequence_header(e, buf + pos);
  pos += write_frame_obu(e, tile, tileSize, buf + pos);
  free(tile);
  e->last.t_entropy += now() - t3;
  e->last.bytes = pos;
  if (!e->nonref) {
    Buf tmp = e->ref;
    e->ref = e->rec;
    e->rec = tmp;
    e->last_id = e->frame_num;
    if (e->cfg.multi_ref && (isKey || e->golden_refresh)) {
      memcpy(e->gold.base, e->ref.base, e->frame_bytes);
      e->gold_id = e->frame_num;
    }
  }
  e->have_ref = 1;
  e->frame_num++;
  e->order_hint++;
  *out = buf;
  *outSize = pos;
  return 0;
}

/* encoder.c:877-915 */
static void copy_out(const Mav1Encoder *e, const uint8_t *frame, uint8_t *const planes[3], const int strides[3]) {
  for (int p = 0; p < 3; p++) {
    int pw = p ? (e->w + 1) >> 1 : e->w;
    int ph = p ? (e->h + 1) >> 1 : e->h;
    for (int y = 0; y < ph; y++)
      memcpy(planes[p] + (size_t)y * strides[p], frame + e->offset[p] + (size_t)y * e->stride[p], pw);
  }
}

static size_t packed_size(const Mav1Encoder *e) {
  size_t cw = (size_t)(e->w + 1) >> 1, ch = (size_t)(e->h + 1) >> 1;
  return (size_t)e->w * e->h + 2 * cw * ch;
}

void mav1_get_recon(const Mav1Encoder *e, uint8_t *const planes[3], const int strides[3]) {
  if (e->cfg.altref > 0) {
    int cw = (e->w + 1) >> 1, ch = (e->h + 1) >> 1;
    const uint8_t *s = e->shown_recon;
    if (!s) return;
    const uint8_t *src[3] = {s, s + (size_t)e->w * e->h, s + (size_t)e->w * e->h + (size_t)cw * ch};
    for (int p = 0; p < 3; p++) {
      int pw = p ? cw : e->w, ph = p ? ch : e->h;
      for (int y = 0; y < ph; y++) memcpy(planes[p] + (size_t)y * strides[p], src[p] + (size_t)y * pw, pw);
    }
    return;
  }
  copy_out(e, e->nonref ? e->rec.base : e->ref.base, planes, strides);
}

/* ---- ALTREF mini-GOPs (encoder.c:917-1293, serial mode) ------------------ */

static int rel_dist(int a, int b) {
  int d = (a - b) & ((1 << 7) - 1);
  return d >= 64 ? d - 128 : d;
}

typedef struct {
  uint8_t *buf;
  size_t pos, cap;
  Mav1FrameStats st;
} Tu;

static void tu_reserve(Tu *t, size_t n) {
  if (t->pos + n > t->cap) {
    t->cap = t->pos + n;
    t->buf = realloc(t->buf, t->cap);
  }
}

static Tu *tu_new(int frameType, int omitTd) {
  Tu *t = calloc(1, sizeof *t);
  t->cap = 1024;
  t->buf = malloc(t->cap);
  if (!omitTd) t->pos = write_temporal_delimiter(t->buf);
  t->st.frame_type = frameType;
  return t;
}

static void alt_push(Mav1Encoder *e, uint8_t *data, size_t size, uint8_t *recon, const Mav1FrameStats *st) {
  if (e->out_n == e->out_cap) {
    e->out_cap = e->out_cap ? 2 * e->out_cap : 8;
    e->outq = realloc(e->outq, sizeof(*e->outq) * e->out_cap);
  }
  struct AltPacket *p = &e->outq[e->out_n++];
  p->data = data;
  p->size = size;
  p->recon = recon;
  p->st = *st;
  p->st.bytes = size;
}

static void tu_close(Mav1Encoder *e, Tu *t, uint8_t *recon) {
  alt_push(e, t->buf, t->pos, recon, &t->st);
  free(t);
}

static void tu_show_existing(Mav1Encoder *e, Tu *t, int slot, uint8_t *recon) {
  tu_reserve(t, 64);
  t->pos += write_show_existing(slot, t->buf + t->pos);
  tu_close(e, t, recon);
}

static void stats_add(Mav1FrameStats *a, const Mav1FrameStats *b) {
  a->num_blocks += b->num_blocks;
  a->num_inter_blocks += b->num_inter_blocks;
  for (int k = 0; k < 16; k++) a->tool_use[k] += b->tool_use[k];
  a->t_analysis += b->t_analysis;
  a->t_recon += b->t_recon;
  a->t_filter += b->t_filter;
  a->t_entropy += b->t_entropy;
}

/* encoder.c:1004-1226 with E == e and every queued job run inline */
static uint8_t *alt_code(Mav1Encoder *e, uint8_t **framep, int disp, int isKey, int kind, int lastSlot, int arfSlot,
                         int refresh, int hidden, Tu *t) {
  if (isKey) e->key_disp = disp;
  e->nonref = e->cfg.leaf && !isKey && refresh == 0;
  e->leafopt = e->nonref ? e->leafopt_cfg : 0;
  e->frame_kind = isKey ? 0 : kind;
  e->order_hint = disp - e->key_disp;
  FrameHdr *h = &e->hdr;
  memset(h, 0, sizeof(*h));
  h->frame_type = isKey ? KEY_FRAME : INTER_FRAME;
  h->base_q_idx = frame_qindex(e, isKey);
  h->order_hint = e->order_hint;
  h->show_frame = !hidden;
  h->showable_frame = hidden;
  h->refresh_frame_flags = isKey ? 0xFF : refresh;
  memset(e->sign_bias, 0, sizeof e->sign_bias);
  if (!isKey) {
    for (int i = 0; i < REFS_PER_FRAME; i++) h->ref_idx[i] = lastSlot;
    if (arfSlot >= 0) h->ref_idx[ALTREF_FRAME - LAST_FRAME] = arfSlot;
    for (int i = 0; i < REFS_PER_FRAME; i++)
      e->sign_bias[LAST_FRAME + i] = rel_dist(e->slot_hint[h->ref_idx[i]], h->order_hint) > 0;
    h->reference_select = kind >= 2 && arfSlot >= 0 && !getenv("MAV1_NOCOMP");
    h->skip_mode_allowed = h->reference_select;
  }
  int rf = h->refresh_frame_flags;
  int lastHint = isKey ? -1 : e->slot_hint[lastSlot], arfHint = !isKey && arfSlot >= 0 ? e->slot_hint[arfSlot] : -1;
  if (rf) e->gen++;
  for (int k = 0; k < 8; k++)
    if ((rf >> k) & 1) {
      e->slot_gen[k] = e->gen;
      e->slot_hint[k] = h->order_hint;
    }
  uint8_t *frame = *framep;
  *framep = NULL;
  int cw = (e->w + 1) >> 1, ch = (e->h + 1) >> 1;
  uint8_t *recon = malloc(packed_size(e));
  /* setup (encoder.c:1088-1118) */
  e->dump_last_hint = lastHint;
  e->dump_arf_hint = arfHint;
  const uint8_t *pl[3] = {frame, frame + (size_t)e->w * e->h, frame + (size_t)e->w * e->h + (size_t)cw * ch};
  int st[3] = {e->w, cw, cw};
  load_source(e, pl, st);
  free(frame);
  if (!isKey) {
    memcpy(e->ref.base, e->slot[lastSlot].base, e->frame_bytes);
    if (arfSlot >= 0) memcpy(e->gold.base, e->slot[arfSlot].base, e->frame_bytes);
  }
  /* core (encoder.c:1121-1149) */
  memset(&e->last, 0, sizeof e->last);
  run_frame_core(e, isKey);
  Mav1FrameStats jst = e->last;
  for (int k = 0; k < 8; k++)
    if ((rf >> k) & 1)
      if (e->slot[k].base) memcpy(e->slot[k].base, e->rec.base, e->frame_bytes);
  uint8_t *rp[3] = {recon, recon + (size_t)e->w * e->h, recon + (size_t)e->w * e->h + (size_t)cw * ch};
  int rs[3] = {e->w, cw, cw};
  copy_out(e, e->rec.base, rp, rs);
  /* tail and append (encoder.c:1194-1224) */
  uint8_t *tile = NULL;
  size_t tileSize = frame_tail(e, &tile, &jst);
  double t3 = now();
  tu_reserve(t, tileSize + 1024);
  if (isKey) {
    t->pos += write_temporal_delimiter(t->buf + t->pos);
    t->pos += write_sequence_header(e, t->buf + t->pos);
  }
  t->pos += write_frame_obu(e, tile, tileSize, t->buf + t->pos);
  free(tile);
  jst.t_entropy += now() - t3;
  stats_add(&t->st, &jst);
  return recon;
}

/* encoder.c:1232-1249 */
static Tu *pyr_code(Mav1Encoder *e, Tu *t, int a, int as, int b, int bs, int depth) {
  int d0 = e->in_disp - e->inq_n;
  if (b - a - 1 >= 3 && depth < 4) {
    int m = (a + b) / 2, ms = 4 + depth;
    if (!t) t = tu_new(1, 0);
    uint8_t *rec = alt_code(e, &e->inq[m - d0], m, 0, 3, as, bs, 1 << ms, 1, t);
    t = pyr_code(e, t, a, as, m, ms, depth + 1);
    if (!t) t = tu_new(1, 0);
    tu_show_existing(e, t, ms, rec);
    return pyr_code(e, NULL, m, ms, b, bs, depth + 1);
  }
  for (int d = a + 1; d < b; d++) {
    if (!t) t = tu_new(1, 0);
    tu_close(e, t, alt_code(e, &e->inq[d - d0], d, 0, 2, as, bs, 0, 0, t));
    t = NULL;
  }
  return t;
}

/* encoder.c:1252-1293 */
static void alt_drain(Mav1Encoder *e, int flush) {
  int N = e->cfg.altref;
  while (e->inq_n > 0) {
    int d0 = e->in_disp - e->inq_n;
    int isKey = d0 == 0 || (e->cfg.keyint > 0 && d0 % e->cfg.keyint == 0);
    int L = isKey ? 1 : N;
    if (!isKey && e->cfg.keyint > 0) L = k_min(L, (d0 / e->cfg.keyint + 1) * e->cfg.keyint - d0);
    if (e->inq_n < L) {
      if (!flush) return;
      L = e->inq_n;
    }
    if (isKey || L == 1) {
      Tu *t = tu_new(!isKey, isKey);
      uint8_t *rec = alt_code(e, &e->inq[0], d0, isKey, 0, e->anchor_slot, -1, 0x01, 0, t);
      e->anchor_slot = 0;
      tu_close(e, t, rec);
    } else if (e->cfg.leaf) {
      int arfSlot = e->anchor_slot == 2 ? 3 : 2;
      Tu *t = tu_new(1, 0);
      uint8_t *arfRecon = alt_code(e, &e->inq[L - 1], d0 + L - 1, 0, 1, e->anchor_slot, -1, 1 << arfSlot, 1, t);
      t = pyr_code(e, t, d0 - 1, e->anchor_slot, d0 + L - 1, arfSlot, 0);
      if (!t) t = tu_new(1, 0);
      tu_show_existing(e, t, arfSlot, arfRecon);
      e->anchor_slot = arfSlot;
    } else {
      int arfSlot = e->anchor_slot == 2 ? 3 : 2;
      Tu *t = tu_new(1, 0);
      uint8_t *arfRecon = alt_code(e, &e->inq[L - 1], d0 + L - 1, 0, 1, e->anchor_slot, -1, 1 << arfSlot, 1, t);
      for (int i = 0; i < L - 1; i++) {
        if (i > 0) t = tu_new(1, 0);
        tu_close(e, t, alt_code(e, &e->inq[i], d0 + i, 0, 2, i == 0 ? e->anchor_slot : 0, arfSlot, 0x01, 0, t));
      }
      t = tu_new(1, 0);
      tu_show_existing(e, t, arfSlot, arfRecon);
      e->anchor_slot = arfSlot;
    }
    for (int i = 0; i < L; i++) free(e->inq[i]);
    memmove(e->inq, e->inq + L, sizeof(*e->inq) * (e->inq_n - L));
    e->inq_n -= L;
  }
}

/* encoder.c:1295-1320 */
int mav1_send_frame(Mav1Encoder *e, const uint8_t *const planes[3], const int strides[3]) {
  if (e->cfg.altref <= 0) {
    if (!planes) return 0;
    if (e->pending) free(e->pend_data);
    e->pending = 1;
    return mav1_encode(e, planes, strides, &e->pend_data, &e->pend_size);
  }
  if (planes) {
    uint8_t *f = malloc(packed_size(e));
    int cw = (e->w + 1) >> 1, ch = (e->h + 1) >> 1;
    for (int p = 0; p < 3; p++) {
      int pw = p ? cw : e->w, ph = p ? ch : e->h;
      uint8_t *d = f + (p ? (size_t)e->w * e->h + (p - 1) * (size_t)cw * ch : 0);
      for (int y = 0; y < ph; y++) memcpy(d + (size_t)y * pw, planes[p] + (size_t)y * strides[p], pw);
    }
    e->inq[e->inq_n++] = f;
    e->in_disp++;
  }
  if (!planes) e->flushing = 1;
  alt_drain(e, planes == NULL);
  return 0;
}

/* encoder.c:1322-1349 */
int mav1_receive_packet(Mav1Encoder *e, uint8_t **out, size_t *outSize) {
  if (e->cfg.altref <= 0) {
    if (!e->pending) return 1;
    e->pending = 0;
    *out = e->pend_data;
    *outSize = e->pend_size;
    return 0;
  }
  if (e->out_pos == e->out_n) {
    e->out_pos = e->out_n = 0;
    return 1;
  }
  struct AltPacket p = e->outq[e->out_pos++];
  *out = p.data;
  *outSize = p.size;
  free(e->shown_recon);
  e->shown_recon = p.recon;
  e->last = p.st;
  return 0;
}

/* encoder.c:1351-1396 (no writer queue: nothing arrives while waiting) */
int mav1_busy(Mav1Encoder *e) { return e->inq_n > 0 || e->pending; }

int mav1_pending_packets(Mav1Encoder *e) {
  if (e->cfg.altref <= 0) return e->pending ? 1 : 0;
  return e->out_n - e->out_pos;
}

int mav1_receive_packet_wait(Mav1Encoder *e, uint8_t **out, size_t *outSize, int timeout_ms) {
  (void)timeout_ms;
  return mav1_receive_packet(e, out, outSize);
}

/* ---- raw access for the tests ---------------------------------------------- */

enum {
  OREF_BUF_SRC, OREF_BUF_REC, OREF_BUF_REF, OREF_BUF_GOLD, OREF_BUF_PARAMS, OREF_BUF_MATS, OREF_BUF_MVFIELD,
  OREF_BUF_MVGOLD, OREF_BUF_BLOCKS, OREF_BUF_SBS, OREF_BUF_COEFS, OREF_BUF_LFMASK, OREF_BUF_CDEFBUF,
  OREF_BUF_DBK, OREF_BUF_LROUT, OREF_BUF_LRUNITS, OREF_BUF_ACOSTS, OREF_BUF_AINFOS, OREF_BUF_HPEL,
  OREF_BUF_CDEF_CHOICE, OREF_BUF_COUNT
};

void *oref_buf(Mav1Encoder *e, int which, size_t *size) {
  Buf *b = NULL;
  switch (which) {
    case OREF_BUF_SRC: b = &e->src; break;
    case OREF_BUF_REC: b = &e->rec; break;
    case OREF_BUF_REF: b = &e->ref; break;
    case OREF_BUF_GOLD: b = &e->gold; break;
    case OREF_BUF_PARAMS: b = &e->params; break;
    case OREF_BUF_MATS: b = &e->mats; break;
    case OREF_BUF_MVFIELD: b = &e->mvfield; break;
    case OREF_BUF_MVGOLD: b = &e->mvgold; break;
    case OREF_BUF_BLOCKS: b = &e->blocks; break;
    case OREF_BUF_SBS: b = &e->sbs; break;
    case OREF_BUF_COEFS: b = &e->coefs; break;
    case OREF_BUF_LFMASK: b = &e->lfmask; break;
    case OREF_BUF_CDEFBUF: b = &e->cdefbuf; break;
    case OREF_BUF_DBK: b = &e->dbk; break;
    case OREF_BUF_LROUT: b = &e->lrout; break;
    case OREF_BUF_LRUNITS: b = &e->lrunits; break;
    case OREF_BUF_ACOSTS: b = &e->acosts; break;
    case OREF_BUF_AINFOS: b = &e->ainfos; break;
    case OREF_BUF_HPEL: b = &e->hpel; break;
    case OREF_BUF_CDEF_CHOICE:
      if (size) *size = (size_t)e->num_sbs;
      return e->cdef_choice;
    default: return NULL;
  }
  if (size) *size = b->size;
  return b->base;
}

/* geometry: w h mi_cols mi_rows sb_cols sb_rows num_sbs tile_cols tile_w_sb
 * frame_bytes num_cdef_presets stride0 stride1 offset1 offset2 */
void oref_geometry(const Mav1Encoder *e, int64_t *g) {
  g[0] = e->w; g[1] = e->h; g[2] = e->mi_cols; g[3] = e->mi_rows; g[4] = e->sb_cols; g[5] = e->sb_rows;
  g[6] = e->num_sbs; g[7] = e->tile_cols; g[8] = e->tile_w_sb; g[9] = (int64_t)e->frame_bytes;
  g[10] = e->num_cdef_presets; g[11] = e->stride[0]; g[12] = e->stride[1]; g[13] = e->offset[1];
  g[14] = e->offset[2];
}

/* Per-frame state the hook sees besides the buffers: frame kind, nonref,
 * leafopt, order hint, key flag, base_q_idx. */
void oref_frame_state(const Mav1Encoder *e, int32_t *s) {
  s[0] = e->frame_kind; s[1] = e->nonref; s[2] = e->leafopt; s[3] = e->order_hint;
  s[4] = e->hdr.frame_type == KEY_FRAME; s[5] = e->hdr.base_q_idx; s[6] = e->num_cdef_presets;
  s[7] = e->hdr.cdef_bits; s[8] = e->hdr.reference_select;
}

/* Layout checks for the product's mirrored structs. */
void oref_struct_sizes(int32_t *s) {
  s[0] = (int32_t)sizeof(FrameParams);
  s[1] = (int32_t)sizeof(BlockInfo);
  s[2] = (int32_t)sizeof(SbInfo);
  s[3] = (int32_t)sizeof(LrUnit);
  s[4] = (int32_t)offsetof(FrameParams, turbo);
  s[5] = (int32_t)offsetof(FrameParams, lr_unit_off);
  s[6] = (int32_t)offsetof(BlockInfo, mv1_col);
  s[7] = (int32_t)offsetof(SbInfo, part);
}

/* Direct stage runners over an encoder whose buffers the caller filled (CPU
 * backend, reference kernels): used by the CPU baseline timing. */
void oref_run_stage(Mav1Encoder *e, int stage) {
  switch (stage) {
    case OREF_STAGE_ME: e->be->motion_search(e->be, e); break;
    case OREF_STAGE_ANALYZE: e->be->analyze(e->be, e); break;
    case OREF_STAGE_EDGE: edge_filter_types(e); break;
    case OREF_STAGE_RECON: e->be->recon(e->be, e); break;
    case OREF_STAGE_FINFO: build_filter_info(e); break;
    case OREF_STAGE_FILTER: e->be->filter(e->be, e); break;
    case OREF_STAGE_CDEFSEL: cdef_select(e); break;
    case OREF_STAGE_LRSEL: lr_select(e); break;
    case OREF_STAGE_RESTORE: e->be->restore(e->be, e); break;
    default: break;
  }
}

void oref_set_num_cdef_presets(Mav1Encoder *e, int n) { e->num_cdef_presets = n; }
