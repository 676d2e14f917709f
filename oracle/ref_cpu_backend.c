/* ORACLE — test infrastructure only; never linked into the product.
 *
 * The reference's CPU backend (src/backend_cpu.c) restated without Apple
 * libdispatch: every dispatch_apply becomes an OpenMP loop over the same work
 * items, calling the reference's own kernels (src/kernels/k_*.h, compiled in
 * place from the reference checkout). Work items of one loop are
 * independent, so the thread count never changes a result.
 *
 * The dependency-counter wavefront of backend_cpu.c:76-156 is restated as
 * waves: superblock (r, c) of a tile column starting at ts runs in wave
 * (c - ts) + 2r, after its left (r, c-1) and above-right (r-1, c+1) (or above,
 * in the tile's last column) neighbours, which lie in earlier waves. */
#include <stdlib.h>

#include "backend.h"
#include "enc_internal.h"
#include "kernels/k_analysis.h"
#include "kernels/k_recon.h"
#include "kernels/k_me.h"
#include "kernels/k_lf.h"
#include "kernels/k_cdef.h"
#include "kernels/k_lr.h"

typedef struct {
  Backend base;
} CpuBackend;

/* backend_cpu.c:23-56 */
static void cpu_motion_search(Backend *b, struct Mav1Encoder *e) {
  (void)b;
  const FrameParams *fp = ENC_PARAMS(e);
  int nref = fp->golden ? 2 : 1;
  uint8_t *qp = e->hpel.base, *srcDec = qp + ME_QP_ENTRIES * qp_entry_bytes(fp);
  if (fp->turbo & T_ME_HPEL) {
    int W = fp->frame_w, H = fp->frame_h;
    long n = (long)H * (nref + 1);
#pragma omp parallel for schedule(dynamic, 4)
    for (long g = 0; g < n; g++) {
      int r = (int)(g / H), y = (int)(g % H);
      for (int x = 0; x < W; x++) {
        int dec = (fp->turbo & T_ME_DEC) && y < dec_h(fp) && x < dec_w(fp);
        if (r == nref) {
          if (dec) dec_build(fp, e->src.base, srcDec, y, x);
          continue;
        }
        uint8_t *ent = qp + r * qp_entry_bytes(fp);
        qpel_build(fp, r ? e->gold.base : e->ref.base, ent, y, x);
        if (dec) dec_build(fp, r ? e->gold.base : e->ref.base, ent + 16L * W * H, y, x);
      }
    }
  }
  for (int level = 0; level < 4; level++) {
    int nn = 1 << (2 * level), nodes = e->num_sbs * nn;
    long n = (long)nodes * nref;
#pragma omp parallel for schedule(dynamic, 8)
    for (long g = 0; g < n; g++) {
      int r = (int)(g / nodes), sb = (int)((g % nodes) / nn), i = (int)(g % nn);
      me_node_serial(fp, sb, level, i, e->src.base, r ? e->gold.base : e->ref.base,
                     qp + r * qp_entry_bytes(fp), srcDec, qp_dec(fp, qp + r * qp_entry_bytes(fp)),
                     (int32_t *)(r ? e->mvgold.base : e->mvfield.base),
                     (int32_t *)e->scratch.base + (size_t)sb * SCRATCH_INTS + r * (SCRATCH_INTS / 2), r);
    }
  }
}

/* backend_cpu.c:58-74 */
void cpu_backend_analyze(Backend *b, struct Mav1Encoder *e) {
  (void)b;
  const FrameParams *fp = ENC_PARAMS(e);
  long *costs = (long *)e->acosts.base;
  BlockInfo *infos = (BlockInfo *)e->ainfos.base;
#pragma omp parallel for schedule(dynamic, 1)
  for (int i = 0; i < e->num_sbs; i++) {
    for (int level = 0; level < 4; level++) {
      int ns = level_slots(fp, level);
      for (int node = 0; node < (1 << (2 * level)); node++)
        for (int slot = 0; slot < ns; slot++)
          analyze_item(fp, i, level, node, slot, e->src.base, e->ref.base, e->gold.base,
                       (const int32_t *)e->mvfield.base, (const int32_t *)e->mvgold.base, costs, infos,
                       (int32_t *)e->scratch.base + (size_t)i * SCRATCH_INTS);
    }
    analyze_sb_table(fp, i, costs, infos, ENC_BLOCKS(e), ENC_SBS(e));
  }
}

/* backend_cpu.c:76-156 as waves (see the file comment). */
void cpu_backend_recon(Backend *b, struct Mav1Encoder *e) {
  (void)b;
  const FrameParams *fp = ENC_PARAMS(e);
  int tw = e->tile_w_sb, waves = tw + 2 * (e->sb_rows - 1);
  int *list = malloc(sizeof(int) * (size_t)e->num_sbs);
  for (int w = 0; w < waves; w++) {
    int n = 0;
    for (int r = 0; r < e->sb_rows; r++)
      for (int c = 0; c < e->sb_cols; c++)
        if ((c % tw) + 2 * r == w) list[n++] = r * e->sb_cols + c;
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = 0; k < n; k++) {
      int idx = list[k];
      recon_sb(fp, ENC_SBS(e)[idx], ENC_BLOCKS(e), e->src.base, e->rec.base, e->ref.base, e->gold.base, ENC_COEFS(e),
               (const int32_t *)e->mats.base, (int32_t *)e->scratch.base + (size_t)idx * SCRATCH_INTS);
    }
  }
  free(list);
}

/* backend_cpu.c:158-177 */
static void cpu_filter(Backend *b, struct Mav1Encoder *e) {
  (void)b;
  const FrameParams *fp = ENC_PARAMS(e);
  const uint8_t *info = e->lfmask.base;
  for (int pass = 0; pass < 2; pass++) {
    int lines = pass == 0 ? e->mi_rows : e->mi_cols;
#pragma omp parallel for schedule(dynamic, 8)
    for (int i = 0; i < 3 * lines; i++) {
      int plane = i / lines, line = i % lines;
      if (plane > 0 && (line & 1)) continue;
      lf_line(fp, e->rec.base, info, plane, pass, line);
    }
  }
  int bc = (e->mi_cols + 1) >> 1, br = (e->mi_rows + 1) >> 1;
  if (e->num_cdef_presets) {
#pragma omp parallel for schedule(dynamic, 16)
    for (int i = 0; i < bc * br; i++)
      cdef_block_all(fp, e->rec.base, e->cdefbuf.base, (long)e->frame_bytes, info, (i / bc) * 2, (i % bc) * 2,
                     e->num_cdef_presets);
  }
}

/* backend_cpu.c:179-188 */
static void cpu_restore(Backend *b, struct Mav1Encoder *e) {
  (void)b;
  const FrameParams *fp = ENC_PARAMS(e);
  int rows4 = (e->h + 3) >> 2, cols4 = (e->w + 3) >> 2, n = rows4 * cols4;
#pragma omp parallel for schedule(dynamic, 64)
  for (int g = 0; g < 3 * n; g++) {
    int plane = g / n, i = g % n;
    lr_block(fp, plane, i / cols4, i % cols4, e->rec.base, e->dbk.base, e->lrout.base,
             (const LrUnit *)e->lrunits.base);
  }
}

static void cpu_destroy(Backend *b) { free(b); }

/* backend_cpu.c:192-203 */
Backend *backend_cpu_create(struct Mav1Encoder *e) {
  (void)e;
  CpuBackend *c = calloc(1, sizeof(*c));
  c->base.name = "cpu";
  c->base.motion_search = cpu_motion_search;
  c->base.analyze = cpu_backend_analyze;
  c->base.recon = cpu_backend_recon;
  c->base.filter = cpu_filter;
  c->base.restore = cpu_restore;
  c->base.destroy = cpu_destroy;
  return &c->base;
}
