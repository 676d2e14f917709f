// Frame driver of the device-resident stream: configuration normalisation,
// the coding order of a clip (key frames, ALTREF mini-GOPs with pyramid
// leaf frames, the plain low-delay path), the per-frame quantizer cascade
// and frame parameters, and the executor that codes one planned frame
// through every device stage with the reference slots kept in HBM.
//
// The frame-structure decisions restate the reference's driver
// (src/encoder.c): create_enc's normalisation :69-112, frame_qindex
// :585-595, setup_params :407-510, run_frame_core's stage gating :599-657,
// mav1_encode :822-875, alt_code :1004-1030, pyr_code :1232-1249 and
// alt_drain :1252-1293. The reference's testing knobs (MAV1_LEAFOPT,
// MAV1_TURBO, MAV1_DT, MAV1_DTB, MAV1_CP, MAV1_Q*, MAV1_NOCOMP,
// MAV1_LEAFINTRA, MAV1_LEAFLF) are read the same way, so both produce the
// same frames under the same environment.
#pragma once

#include <stdlib.h>

#include <vector>

#include "common.cuh"

namespace drv {

static int env_or(const char *n, int d) {
  const char *v = getenv(n);
  return v ? atoi(v) : d;
}

struct Norm {
  mav1cu_config c;
  int leafopt_cfg;
  int mi_cols, mi_rows, sb_cols, sb_rows, tile_w_sb, tile_cols;
  int tile_cols_log2, min_log2_tile_cols, max_log2_tile_cols;
};

static Norm normalise(const mav1cu_config *in) {
  Norm n;
  n.c = *in;
  mav1cu_config &c = n.c;
  if (c.turbo) {
    c.fast = 1;
    if (c.altref < 2) c.altref = 2;
    c.leaf = 1;
  }
  if (c.altref == 1) c.altref = 0;
  if (c.altref > 16) c.altref = 16;
  if (c.altref) c.multi_ref = c.nonref_odd = 0;
  if (!c.altref) c.leaf = 0;
  n.leafopt_cfg = getenv("MAV1_LEAFOPT") ? (int)strtol(getenv("MAV1_LEAFOPT"), NULL, 0) : 0x3F;
  if (c.qindex < 0) c.qindex = 0;
  if (c.qindex > 255) c.qindex = 255;
  n.mi_cols = 2 * ((c.width + 7) >> 3);
  n.mi_rows = 2 * ((c.height + 7) >> 3);
  n.sb_cols = (n.mi_cols + 15) >> 4;
  n.sb_rows = (n.mi_rows + 15) >> 4;
  int k = 0;
  while (((4096 >> 6) << k) < n.sb_cols) k++;
  int minLog2 = k;
  int maxCols = n.sb_cols < 64 ? n.sb_cols : 64;
  for (k = 0; (1 << k) < maxCols; k++) {
  }
  int maxLog2 = k;
  int l = c.tile_cols_log2;
  if (l < minLog2) l = minLog2;
  if (l > maxLog2) l = maxLog2;
  n.tile_w_sb = (n.sb_cols + (1 << l) - 1) >> l;
  n.tile_cols = (n.sb_cols + n.tile_w_sb - 1) / n.tile_w_sb;
  n.tile_cols_log2 = l;
  n.min_log2_tile_cols = minLog2;
  n.max_log2_tile_cols = maxLog2;
  return n;
}

// Quantizer cascade (encoder.c:585-595).
static int frame_q(const Norm &n, int isKey, int orderHint, int nonref, int kind) {
  int q = n.c.qindex;
  if (q == 0) return 0;
  int off = isKey ? env_or("MAV1_QK", -24) : (orderHint % 4 == 0 ? env_or("MAV1_Q4", -8) : env_or("MAV1_QP", 4));
  if (!isKey && nonref) off = env_or("MAV1_QN", 12);
  if (!isKey && n.c.altref) off = kind == 1 ? env_or("MAV1_QA", -8) : env_or("MAV1_QP", 4);
  if (!isKey && n.c.leaf && kind == 3) off = env_or("MAV1_QM", 0);
  if (!isKey && n.c.leaf && nonref) off = env_or("MAV1_QL", 8);
  q += off;
  return q < 1 ? 1 : q > 255 ? 255 : q;
}

struct Planner {
  Norm n;
  std::vector<mav1cu_frame_job> jobs;
  // ALTREF driver: display index of the current key frame, the anchor slot,
  // frames received so far and frames received but not yet coded
  int key_disp = 0, anchor_slot = 0, in_disp = 0, inq_n = 0;
  // low-delay driver (mav1_encode): OrderHint and the frames held by LAST /
  // GOLDEN (encoder.c:822-875)
  int ld_order_hint = 0, ld_last_id = 0, ld_gold_id = 0;

  // alt_code's frame-structure part (encoder.c:1004-1030)
  void code(int disp, int isKey, int kind, int lastSlot, int arfSlot, int refresh, int hidden) {
    mav1cu_frame_job j = {};
    if (isKey) key_disp = disp;
    j.disp = disp;
    j.is_key = isKey;
    j.nonref = n.c.leaf && !isKey && refresh == 0;
    j.leafopt = j.nonref ? n.leafopt_cfg : 0;
    j.kind = isKey ? 0 : kind;
    j.order_hint = disp - key_disp;
    j.base_q_idx = frame_q(n, isKey, j.order_hint, j.nonref, j.kind);
    j.hidden = hidden;
    j.refresh = isKey ? 0xFF : refresh;
    j.last_slot = isKey ? -1 : lastSlot;
    j.arf_slot = isKey ? -1 : arfSlot;
    j.reference_select = !isKey && kind >= 2 && arfSlot >= 0 && !getenv("MAV1_NOCOMP");
    j.show_existing = -1;
    jobs.push_back(j);
  }

  // pyr_code (encoder.c:1232-1249)
  void pyr(int a, int as, int b, int bs, int depth) {
    if (b - a - 1 >= 3 && depth < 4) {
      int m = (a + b) / 2, ms = 4 + depth;
      code(m, 0, 3, as, bs, 1 << ms, 1);
      pyr(a, as, m, ms, depth + 1);
      jobs.back().show_existing = ms;
      pyr(m, ms, b, bs, depth + 1);
      return;
    }
    for (int d = a + 1; d < b; d++) code(d, 0, 2, as, bs, 0, 0);
  }

  // alt_drain (encoder.c:1252-1293): codes the queued frames that can be
  // coded, all of them when flushing
  void alt_drain(bool flush) {
    int N = n.c.altref;
    const int keyint = n.c.keyint;
    while (inq_n > 0) {
      int d0 = in_disp - inq_n;
      int isKey = d0 == 0 || (keyint > 0 && d0 % keyint == 0);
      int L = isKey ? 1 : N;
      if (!isKey && keyint > 0) L = imin(L, (d0 / keyint + 1) * keyint - d0);
      if (inq_n < L) {
        if (!flush) return;
        L = inq_n;
      }
      if (isKey || L == 1) {
        code(d0, isKey, 0, anchor_slot, -1, 0x01, 0);
        anchor_slot = 0;
      } else if (n.c.leaf) {
        int arfSlot = anchor_slot == 2 ? 3 : 2;
        code(d0 + L - 1, 0, 1, anchor_slot, -1, 1 << arfSlot, 1);
        pyr(d0 - 1, anchor_slot, d0 + L - 1, arfSlot, 0);
        jobs.back().show_existing = arfSlot;
        anchor_slot = arfSlot;
      } else {
        int arfSlot = anchor_slot == 2 ? 3 : 2;
        code(d0 + L - 1, 0, 1, anchor_slot, -1, 1 << arfSlot, 1);
        for (int i = 0; i < L - 1; i++) code(d0 + i, 0, 2, i == 0 ? anchor_slot : 0, arfSlot, 0x01, 0);
        jobs.back().show_existing = arfSlot;
        anchor_slot = arfSlot;
      }
      inq_n -= L;
    }
  }

  // every frame of a clip queued, then the stream flushed
  void drain(int nframes) {
    in_disp = nframes;
    inq_n = nframes;
    alt_drain(true);
  }

  // mav1_encode's frame structure for the next frame (encoder.c:822-875):
  // LAST in slot 0, GOLDEN in slot 1
  void low_delay_frame() {
    mav1cu_frame_job j = {};
    int f = in_disp++;
    int isKey = f == 0 || (n.c.keyint > 0 && f % n.c.keyint == 0);
    j.disp = f;
    j.is_key = isKey;
    j.nonref = !isKey && n.c.nonref_odd && (ld_order_hint & 1);
    j.base_q_idx = frame_q(n, isKey, ld_order_hint, j.nonref, 0);
    if (isKey) ld_order_hint = 0;
    j.order_hint = ld_order_hint;
    j.golden_refresh = !isKey && !j.nonref && n.c.multi_ref && ld_order_hint % 4 == 0;
    j.refresh = isKey ? 0xFF : (j.nonref ? 0x00 : 0x01 | (j.golden_refresh ? 0x02 : 0));
    j.last_slot = isKey ? -1 : 0;
    j.arf_slot = isKey || !n.c.multi_ref ? -1 : 1;
    j.gold_differs = ld_gold_id != ld_last_id;
    j.show_existing = -1;
    jobs.push_back(j);
    if (!j.nonref) {
      ld_last_id = f;
      if (n.c.multi_ref && (isKey || j.golden_refresh)) ld_gold_id = f;
    }
    ld_order_hint++;
  }

  void low_delay(int nframes) {
    for (int f = 0; f < nframes; f++) low_delay_frame();
  }

  // the caller-held state of an incremental plan (mav1cu_planner)
  void load(const mav1cu_planner &p) {
    key_disp = p.key_disp;
    anchor_slot = p.anchor_slot;
    in_disp = p.in_disp;
    inq_n = p.inq_n;
    ld_order_hint = p.ld_order_hint;
    ld_last_id = p.ld_last_id;
    ld_gold_id = p.ld_gold_id;
  }
  void store(mav1cu_planner *p) const {
    p->key_disp = key_disp;
    p->anchor_slot = anchor_slot;
    p->in_disp = in_disp;
    p->inq_n = inq_n;
    p->ld_order_hint = ld_order_hint;
    p->ld_last_id = ld_last_id;
    p->ld_gold_id = ld_gold_id;
  }
};

// setup_params (encoder.c:407-510) for one planned frame.
static void frame_params(const Norm &n, const mav1cu_frame_job &j, FrameParams *fp, int *presets) {
  const mav1cu_config &c = n.c;
  memset(fp, 0, sizeof(*fp));
  int isKey = j.is_key;
  fp->mi_cols = n.mi_cols;
  fp->mi_rows = n.mi_rows;
  fp->sb_cols = n.sb_cols;
  fp->sb_rows = n.sb_rows;
  int stride0 = n.sb_cols * 64, stride1 = n.sb_cols * 32, ph0 = n.sb_rows * 64, ph1 = n.sb_rows * 32;
  int strides[3] = {stride0, stride1, stride1}, phs[3] = {ph0, ph1, ph1};
  int offs[3] = {0, stride0 * ph0, stride0 * ph0 + stride1 * ph1};
  for (int p = 0; p < 3; p++) {
    fp->plane_w[p] = strides[p];
    fp->plane_h[p] = phs[p];
    fp->stride[p] = strides[p];
    fp->offset[p] = offs[p];
  }
  int q = j.base_q_idx;
  fp->base_q_idx = q;
  for (int p = 0; p < 3; p++) {
    fp->dc_q[p] = h_Dc_Qlookup[0][q];
    fp->ac_q[p] = h_Ac_Qlookup[0][q];
  }
  fp->frame_is_intra = isKey;
  fp->reduced_tx_set = 0;
  fp->enable_intra_edge_filter = c.intra_edge_filter;
  fp->tx_search = c.tx_search;
  fp->lossless = q == 0;
  fp->tx_mode_select = q != 0 && c.tx_depth;
  fp->switchable_interp = !isKey && c.switchable_interp;
  fp->golden = !isKey && c.multi_ref && j.gold_differs;
  fp->ref2_frame = GOLDEN_FRAME;
  if (c.altref) {
    fp->golden = !isKey && j.kind >= 2;
    fp->ref2_frame = ALTREF_FRAME;
    fp->compound = j.reference_select;
  }
  fp->fast = c.fast;
  fp->turbo = c.turbo ? (getenv("MAV1_TURBO") ? (int)strtol(getenv("MAV1_TURBO"), NULL, 0) : 0x47CBF1) : 0;
  fp->leaf = c.leaf ? (j.leafopt & 1) : j.nonref && !getenv("MAV1_LEAFINTRA");
  if (j.leafopt & 16) fp->tx_search = 0;
  {
    int dt = getenv("MAV1_DT") ? atoi(getenv("MAV1_DT")) : n.sb_rows >= 16 ? 320 : 352;
    int bias = getenv("MAV1_DTB") ? atoi(getenv("MAV1_DTB")) : 0;
    fp->depth_thr = c.turbo ? dt * (q + bias) / (128 + bias) : 0;
  }
  fp->tile_w_sb = n.tile_w_sb;
  long long acq = fp->ac_q[0];
  fp->lambda = (int32_t)(acq * acq * 256 / 430);
  fp->frame_w = c.width;
  fp->frame_h = c.height;
  fp->me_range = c.me_range;
  if ((j.leafopt & 32) && fp->me_range > 16) fp->me_range = 16;
  int lvl = 0;
  if (c.loop_filter && q > 0 && !(c.leaf ? (j.leafopt & 2) : j.nonref && !getenv("MAV1_LEAFLF"))) {
    lvl = (int)((acq * 20723 + 1015158 + (1 << 17)) >> 18);
    if (!isKey) lvl -= 4;
    lvl = lvl < 0 ? 0 : (lvl > MAX_LOOP_FILTER ? MAX_LOOP_FILTER : lvl);
  }
  for (int i = 0; i < 4; i++) fp->lf_level[i] = lvl;
  fp->lf_sharpness = 0;
  static const int presetTab[4][4] = {{0, 0, 0, 0}, {2, 1, 1, 0}, {4, 2, 2, 1}, {8, 4, 4, 2}};
  fp->cdef_damping = 3 + (q >> 6);
  fp->cdef_bits = 2;
  if (j.leafopt & 4) {
    fp->cdef_damping = 3;
    fp->cdef_bits = 0;
  }
  int pi[4] = {0, 1, 2, 3};
  if ((fp->turbo & 2048) && fp->cdef_bits == 2) {
    fp->cdef_bits = 1;
    pi[1] = env_or("MAV1_CP", 2);
  }
  for (int i = 0; i < 4; i++) {
    const int *ps = presetTab[pi[i]];
    fp->cdef_y_pri[i] = ps[0];
    fp->cdef_y_sec[i] = ps[1];
    fp->cdef_uv_pri[i] = ps[2];
    fp->cdef_uv_sec[i] = ps[3];
  }
  int off = 0;
  for (int p = 0; p < 3; p++) {
    int sub = p > 0, size = 256 >> 2;
    int pw = (c.width + sub) >> sub, ph = (c.height + sub) >> sub;
    fp->lr_type[p] = RESTORE_NONE;
    fp->lr_unit_size[p] = size;
    fp->lr_unit_rows[p] = imax((ph + (size >> 1)) / size, 1);
    fp->lr_unit_cols[p] = imax((pw + (size >> 1)) / size, 1);
    fp->lr_unit_off[p] = off;
    off += fp->lr_unit_rows[p] * fp->lr_unit_cols[p];
  }
  // presets the filter stage writes (run_frame_core, encoder.c:625-632)
  int nPresets = c.cdef ? 4 : 0, cdefOff = (j.leafopt & 4) != 0;
  *presets = cdefOff ? 0 : (nPresets ? 1 << fp->cdef_bits : 0);
}

// Stores frame parameters passed by value (the launch copies them).
__global__ void k_store_params(FrameParams fp, FrameParams *dst) {
  const int *a = (const int *)&fp;
  int *d = (int *)dst;
  for (int k = threadIdx.x; k < (int)(sizeof(FrameParams) / 4); k += blockDim.x) d[k] = a[k];
}

// load_source (encoder.c:297-310): the I420 picture into the padded planar
// layout, the right and bottom edges replicated up to the superblock-aligned
// size. A thread writes 16 consecutive samples of a row as one 16-byte store
// (padded rows are multiples of 32 samples, plane offsets multiples of 1024)
// and reads them as one 16-byte load where the source run is aligned and
// inside the row, byte by byte with the edge clamp otherwise. CTAs of 32 x 8
// threads cover 512 samples of 8 rows; blockIdx.z is the plane.
constexpr int LS_ROWS = 8;
__global__ void __launch_bounds__(256) k_load_source(const uint8_t *i420, uint8_t *dst, int w, int h, int sbCols,
                                                     int sbRows) {
  int p = blockIdx.z;
  int pw = p ? (w + 1) >> 1 : w, ph = p ? (h + 1) >> 1 : h;
  int aw = p ? sbCols * 32 : sbCols * 64, ah = p ? sbRows * 32 : sbRows * 64;
  int x = (blockIdx.x * 32 + threadIdx.x) * 16, y = blockIdx.y * LS_ROWS + threadIdx.y;
  if (x >= aw || y >= ah) return;
  size_t planeOff = p == 0 ? 0 : (size_t)w * h + (size_t)(p - 1) * ((w + 1) >> 1) * ((h + 1) >> 1);
  size_t dstOff = p == 0 ? 0 : (size_t)sbCols * 64 * sbRows * 64 + (size_t)(p - 1) * sbCols * 32 * sbRows * 32;
  const uint8_t *row = i420 + planeOff + (size_t)imin(y, ph - 1) * pw;
  uint4 v;
  if (x + 16 <= pw && (((uintptr_t)(row + x)) & 15) == 0) {
    v = *(const uint4 *)(row + x);
  } else {
    uint8_t b[16];
#pragma unroll
    for (int k = 0; k < 16; k++) b[k] = row[imin(x + k, pw - 1)];
    v = make_uint4(b[0] | b[1] << 8 | b[2] << 16 | (unsigned)b[3] << 24, b[4] | b[5] << 8 | b[6] << 16 | (unsigned)b[7] << 24,
                   b[8] | b[9] << 8 | b[10] << 16 | (unsigned)b[11] << 24,
                   b[12] | b[13] << 8 | b[14] << 16 | (unsigned)b[15] << 24);
  }
  *(uint4 *)(dst + dstOff + (size_t)y * aw + x) = v;
}

}  // namespace drv
