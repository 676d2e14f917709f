/* The reference's entropy coder and OBU writer over the writer inputs that
 * the device exports.
 *
 * Entropy coding and OBU assembly stay the reference encoder's host code:
 * src/tile_writer.c (compiled here, in place, through the #include below),
 * src/mvpred.c, src/entenc.c, src/cdfs.c, src/bitwriter.c, src/obu.c and the
 * rate coding of loop-restoration units in src/lr_search.c are linked
 * unchanged. They read the encoder's internal state (struct Mav1Encoder of
 * src/enc_internal.h); this file fills one such "writer view" per context
 * with exactly the fields they read: the normalised configuration and
 * geometry (create_enc, encoder.c:69-120), the frame header (FrameHdr), the
 * sign bias of the references, the MiInfo grid and CDEF indices they fill
 * while coding, and the BLOCKS / SBS / COEFS / CDEF choice / LR unit
 * buffers, which point into the export image.
 *
 * tile_writer.c's one libdispatch statement (the dispatch_apply over tile
 * columns in write_tile, tile_writer.c:610, a clang Blocks literal that gcc
 * cannot parse) is swallowed by the macro below, and write_tile itself is
 * renamed out of the way: the host driver runs its steps itself (the
 * set-up, then write_one_tile per column on its thread pool, then the
 * concatenation), so the tile columns of a frame code concurrently as in the
 * reference. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define dispatch_apply(...) ((void)0)
#define write_tile mh_reference_write_tile_unused
#include "tile_writer.c"
#undef write_tile
#undef dispatch_apply

#include "mh_writer.h"

_Static_assert(sizeof(Mav1Config) == sizeof(mav1cu_config), "Mav1Config layout");
_Static_assert(sizeof(FrameParams) == sizeof(mav1cu_frame_params), "FrameParams layout");
_Static_assert(sizeof(BlockInfo) == sizeof(mav1cu_block_info), "BlockInfo layout");
_Static_assert(sizeof(SbInfo) == sizeof(mav1cu_sb_info), "SbInfo layout");
_Static_assert(sizeof(LrUnit) == sizeof(mav1cu_lr_unit), "LrUnit layout");

struct mh_writer {
  struct Mav1Encoder e;    /* the writer view */
  const mav1cu_frame_job *job;
  int low_delay;
  int last_hint, arf_hint;
  size_t lr_bytes;
  void *lr_zero;           /* LR units of frames without loop restoration */
};

mh_writer *mh_writer_new(const mav1cu_layout *L) {
  mh_writer *w = calloc(1, sizeof *w);
  if (!w) return NULL;
  struct Mav1Encoder *e = &w->e;
  memcpy(&e->cfg, &L->cfg, sizeof e->cfg);
  e->w = L->cfg.width;
  e->h = L->cfg.height;
  e->mi_cols = L->mi_cols;
  e->mi_rows = L->mi_rows;
  e->sb_cols = L->sb_cols;
  e->sb_rows = L->sb_rows;
  e->num_sbs = L->num_sbs;
  e->tile_cols_log2 = L->tile_cols_log2;
  e->tile_cols = L->tile_cols;
  e->tile_w_sb = L->tile_w_sb;
  e->min_log2_tile_cols = L->min_log2_tile_cols;
  e->max_log2_tile_cols = L->max_log2_tile_cols;
  for (int p = 0; p < 3; p++) {
    e->stride[p] = L->stride[p];
    e->offset[p] = L->offset[p];
    e->plane_h[p] = L->plane_h[p];
  }
  e->frame_bytes = (size_t)L->frame_bytes;
  e->leafopt_cfg = L->leafopt_cfg;
  e->mi = calloc((size_t)e->mi_rows * e->mi_cols, sizeof(MiInfo));
  e->cdef_idx = calloc((size_t)e->num_sbs, 1);
  w->lr_bytes = sizeof(LrUnit) * 3 * (size_t)(e->sb_rows + 1) * (e->sb_cols + 1);
  w->lr_zero = calloc(1, w->lr_bytes);
  if (!e->mi || !e->cdef_idx || !w->lr_zero) {
    mh_writer_free(w);
    return NULL;
  }
  e->num_cdef_presets = 1 << 2;
  return w;
}

void mh_writer_config(mh_writer *w, const mav1cu_layout *L) {
  memcpy(&w->e.cfg, &L->cfg, sizeof w->e.cfg);
  w->e.leafopt_cfg = L->leafopt_cfg;
}

void mh_writer_free(mh_writer *w) {
  if (!w) return;
  free(w->e.mi);
  free(w->e.cdef_idx);
  free(w->lr_zero);
  free(w);
}

static int rel_dist(int a, int b) {
  int d = (a - b) & ((1 << 7) - 1); /* OrderHintBits = 7 */
  return d >= 64 ? d - 128 : d;
}

void mh_writer_frame(mh_writer *w, const mh_frame *f) {
  struct Mav1Encoder *e = &w->e;
  const mav1cu_frame_job *j = f->job;
  const mav1cu_frame_params *fp = f->fp;
  w->job = j;
  w->low_delay = f->low_delay;
  w->last_hint = f->last_hint;
  w->arf_hint = f->arf_hint;
  FrameHdr *h = &e->hdr;
  memset(h, 0, sizeof *h);
  memset(e->sign_bias, 0, sizeof e->sign_bias);
  int isKey = j->is_key;
  h->frame_type = isKey ? KEY_FRAME : INTER_FRAME;
  h->base_q_idx = j->base_q_idx;
  h->order_hint = j->order_hint;
  h->refresh_frame_flags = j->refresh;
  if (f->low_delay) {
    /* mav1_encode (encoder.c:831-846): shown, LAST -> slot 0, GOLDEN -> slot 1 */
    h->show_frame = 1;
    if (e->cfg.multi_ref) h->ref_idx[GOLDEN_FRAME - LAST_FRAME] = 1;
  } else {
    /* alt_code (encoder.c:1013-1030) */
    h->show_frame = !j->hidden;
    h->showable_frame = j->hidden;
    if (!isKey) {
      for (int i = 0; i < REFS_PER_FRAME; i++) h->ref_idx[i] = j->last_slot;
      if (j->arf_slot >= 0) h->ref_idx[ALTREF_FRAME - LAST_FRAME] = j->arf_slot;
      for (int i = 0; i < REFS_PER_FRAME; i++) e->sign_bias[LAST_FRAME + i] = rel_dist(f->ref_hint[i], h->order_hint) > 0;
      h->reference_select = j->reference_select;
      h->skip_mode_allowed = h->reference_select;
    }
  }
  /* header fields setup_params derives with the frame parameters
   * (encoder.c:467-509) */
  for (int i = 0; i < 4; i++) h->lf_level[i] = fp->lf_level[i];
  h->lf_sharpness = fp->lf_sharpness;
  h->cdef_damping = fp->cdef_damping;
  h->cdef_bits = fp->cdef_bits;
  for (int i = 0; i < 8; i++) {
    h->cdef_y_pri[i] = fp->cdef_y_pri[i];
    h->cdef_y_sec[i] = fp->cdef_y_sec[i];
    h->cdef_uv_pri[i] = fp->cdef_uv_pri[i];
    h->cdef_uv_sec[i] = fp->cdef_uv_sec[i];
  }
  for (int p = 0; p < 3; p++) h->lr_type[p] = fp->lr_type[p];
  e->nonref = j->nonref;
  e->leafopt = j->leafopt;
  e->frame_kind = j->kind;
  e->order_hint = j->order_hint;
  e->dump_last_hint = f->last_hint;
  e->dump_arf_hint = f->arf_hint;
  /* the writer inputs */
  e->params.base = (uint8_t *)fp;
  e->params.size = sizeof *fp;
  e->sbs.base = (uint8_t *)f->sbs;
  e->blocks.base = (uint8_t *)f->blocks;
  e->coefs.base = (uint8_t *)f->coefs;
  e->cdef_choice = (int8_t *)f->cdef_choice;
  e->lrunits.base = (uint8_t *)(f->lrunits ? (const void *)f->lrunits : w->lr_zero);
  e->lrunits.size = w->lr_bytes;
}

void mh_writer_begin(mh_writer *w) {
  struct Mav1Encoder *e = &w->e;
  memset(e->mi, 0, sizeof(MiInfo) * e->mi_rows * e->mi_cols);
  for (int i = 0; i < e->num_sbs; i++) e->cdef_idx[i] = -1;
  mvpred_frame_start(e);
}

size_t mh_writer_tile(mh_writer *w, int tc, uint8_t **out) { return write_one_tile(&w->e, tc, out); }
int mh_writer_tile_cols(const mh_writer *w) { return w->e.tile_cols; }

size_t mh_writer_frame_obu(mh_writer *w, const uint8_t *tile, size_t tileSize, uint8_t *out) {
  return write_frame_obu(&w->e, tile, tileSize, out);
}

size_t mh_writer_sequence_header(mh_writer *w, uint8_t *out) { return write_sequence_header(&w->e, out); }
size_t mh_temporal_delimiter(uint8_t *out) { return write_temporal_delimiter(out); }
size_t mh_show_existing(int slot, uint8_t *out) { return write_show_existing(slot, out); }

uint8_t *mh_writer_dump_record(mh_writer *w, size_t tileSize, size_t *bytes) {
  /* one record per coded frame: 11 x int32 header, then an 8-byte cell per
   * 8x8 unit (bsize, mode, ref_frame, 0, Mv[0] row and column as int16);
   * the format of dump_decisions, encoder.c:659-704 */
  const struct Mav1Encoder *s = &w->e;
  int rows8 = (s->mi_rows + 1) >> 1, cols8 = (s->mi_cols + 1) >> 1;
  size_t cells = (size_t)rows8 * cols8;
  uint8_t *rec = calloc(44 + cells * 8, 1);
  if (!rec) return NULL;
  uint8_t *grid = rec + 44;
  const SbInfo *sbs = ENC_SBS(s);
  const BlockInfo *blocks = ENC_BLOCKS(s);
  for (int i = 0; i < s->num_sbs; i++)
    for (int k = 0; k < sbs[i].num_blocks; k++) {
      const BlockInfo *b = &blocks[sbs[i].first_block + k];
      int w8 = (Num_4x4_Blocks_Wide[b->bsize] + 1) >> 1, h8 = (Num_4x4_Blocks_High[b->bsize] + 1) >> 1;
      int r0 = b->mi_row >> 1, c0 = b->mi_col >> 1;
      int16_t mv[2] = {(int16_t)b->mv_row, (int16_t)b->mv_col};
      for (int r = r0; r < r0 + h8 && r < rows8; r++)
        for (int c = c0; c < c0 + w8 && c < cols8; c++) {
          uint8_t *cell = grid + ((size_t)r * cols8 + c) * 8;
          cell[0] = (uint8_t)b->bsize;
          cell[1] = !b->is_inter ? 0 : b->ref_frame1 ? 2 : 1;
          cell[2] = (uint8_t)b->ref_frame;
          cell[3] = 0;
          memcpy(cell + 4, mv, 4);
        }
    }
  int32_t hdr[11] = {0x4345444D, s->order_hint, s->dump_last_hint, s->dump_arf_hint,
                     s->hdr.frame_type == KEY_FRAME ? 0 : 1, s->frame_kind, s->nonref, s->hdr.base_q_idx,
                     rows8, cols8, (int32_t)tileSize};
  memcpy(rec, hdr, sizeof hdr);
  *bytes = 44 + cells * 8;
  return rec;
}

void mh_writer_stats(mh_writer *w, int *numBlocks, int *numInter, int toolUse[16]) {
  const struct Mav1Encoder *s = &w->e;
  const SbInfo *sbs = ENC_SBS(s);
  const BlockInfo *blocks = ENC_BLOCKS(s);
  int nb = 0, ni = 0;
  memset(toolUse, 0, 16 * sizeof(int));
  for (int i = 0; i < s->num_sbs; i++) {
    nb += sbs[i].num_blocks;
    for (int k = 0; k < sbs[i].num_blocks; k++) {
      const BlockInfo *b = &blocks[sbs[i].first_block + k];
      ni += b->is_inter;
      toolUse[0] += !b->is_inter;
      toolUse[1] += b->is_inter;
      toolUse[2] += !b->is_inter && b->uv_mode == UV_CFL_PRED;
      toolUse[3] += !b->is_inter && (b->angle_y != 0 || b->angle_uv != 0);
      toolUse[4] += b->eob[0] > 0 && b->tx_type != DCT_DCT;
      toolUse[5] += b->eob[0] == 0 && b->eob[1] == 0 && b->eob[2] == 0;
      toolUse[6] += Block_Width(b->bsize) != Block_Height(b->bsize);
      toolUse[7] += b->is_inter && b->ref_frame1 > INTRA_FRAME;
      toolUse[11] += b->is_inter && b->ref_frame == GOLDEN_FRAME;
      toolUse[12] += b->is_inter && b->ref_frame == ALTREF_FRAME;
    }
  }
  *numBlocks = nb;
  *numInter = ni;
}
