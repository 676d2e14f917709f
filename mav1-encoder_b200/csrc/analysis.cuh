// Open-loop mode and partition analysis (reference src/kernels/k_analysis.h).
//
// Pass 1 evaluates every candidate block of every superblock independently:
// the inter candidates (LAST, the second reference, their compound average)
// by luma + chroma SATD plus a motion-vector rate, the intra modes by SATD
// of a prediction from the source neighbours plus a mode rate, chroma modes
// and chroma-from-luma, and keeps the cheapest (eval_block,
// k_analysis.h:241-404; analyze_item :656-679). Pass 2 makes the bottom-up
// partition decision per superblock and emits its blocks in decode order
// (analyze_sb_table :697-808).
//
// B200 mapping: one warp per candidate block. Each lane predicts whole 4x4
// units in registers (inter samples through pred::inter_unit4, intra samples
// from edge arrays in the warp's shared memory), so a prediction is never
// materialised; SATD sums are reduced with shuffles. Levels run as separate
// launches 64x64 -> 8x8 because the depth pruning reads the ancestors' costs.
// Pass 2 is one thread per superblock (a few hundred integer comparisons).
#pragma once

#include "common.cuh"
#include "pred.cuh"

namespace ana {

struct Ctx {
  const FrameParams *fp;
  const uint8_t *src, *ref, *gold;
  const int32_t *mv, *mvg;
  int64_t *costs;
  BlockInfo *infos;
  BlockInfo *blocks;
  SbInfo *sbs;
};

#define GOLDEN_REF_BITS8 8
#define COMPOUND_BITS8 16

struct WarpMem {
  int edge[3][2][EDGE_LEN];  // [plane][above / left]
};

__device__ __forceinline__ int warp_sum(int v) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}
__device__ __forceinline__ long long warp_sum64(long long v) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  return v;
}

// The threads evaluating one candidate: a warp (rank = lane), half a warp
// (the 8x8 level: a few 4x4 units per candidate; mask holds its lanes), or
// for the 64x64 level a whole CTA (red: one shared word per warp). Sums are
// the group's lanes' sums, then across the CTA's warps.
struct Grp {
  int rank, size;
  long long *red;
  unsigned mask;
};
__device__ __forceinline__ void gsync(const Grp &g) {
  if (g.size <= 32) __syncwarp(g.mask);
  else __syncthreads();
}
__device__ __forceinline__ long long gsum64(long long v, const Grp &g) {
  if (g.size < 32) {
    for (int off = g.size >> 1; off > 0; off >>= 1) v += __shfl_xor_sync(g.mask, v, off);
    return v;
  }
  v = warp_sum64(v);
  if (g.size == 32) return v;
  __syncthreads();
  if ((g.rank & 31) == 0) g.red[g.rank >> 5] = v;
  __syncthreads();
  long long t = 0;
  for (int k = 0; k < (g.size >> 5); k++) t += g.red[k];
  return t;
}
__device__ __forceinline__ int gsum(int v, const Grp &g) { return (int)gsum64(v, g); }

HD int mode_bits8(int mode) {
  if (mode == DC_PRED) return 12;
  if (mode == V_PRED || mode == H_PRED || mode == SMOOTH_PRED || mode == PAETH_PRED) return 26;
  if (mode == SMOOTH_V_PRED || mode == SMOOTH_H_PRED) return 34;
  return 40;
}
HD int mv_bits8(int mvr, int mvc) {
  return 8 * (2 + 2 * floor_log2(iabs(mvr) + 1) + 2 * floor_log2(iabs(mvc) + 1));
}
HD int turbo_mode_off(const FrameParams *fp, int mode) {
  return (fp->turbo & T_INTRA) && !fp->frame_is_intra && mode != DC_PRED && mode != V_PRED && mode != H_PRED &&
         mode != SMOOTH_PRED;
}
HD int turbo_no_cfl(const FrameParams *fp) { return (fp->turbo & T_INTRA) && !fp->frame_is_intra; }
HD int eval_sub(const FrameParams *fp) { return (fp->turbo & T_ANA_USUB) != 0; }

// ---- inter SATDs --------------------------------------------------------------

// block_satd_e of one plane predicted from one reference (k_analysis.h:113-119):
// checkerboard units x2 when the analysis subsampling is on and bw >= 32.
__device__ int inter_plane_satd(const FrameParams *fp, const uint8_t *src, const uint8_t *ref, int p, int bx, int by,
                                int bw, int bh, int mvr, int mvc, const Grp &g) {
  int sub = p > 0, stride = fp->stride[p];
  pred::Inter ip;
  pred::inter_setup(&ip, ref + fp->offset[p], stride, fp->frame_w, fp->frame_h, bx, by, bw, bh, mvr, mvc, sub, sub,
                    EIGHTTAP);
  const uint8_t *sp = src + fp->offset[p] + by * stride + bx;
  int usub = eval_sub(fp) && bw >= 32 ? 2 : 1;
  int nux = bw >> 2, nu = nux * (bh >> 2), s = 0;
  for (int u = g.rank; u < nu; u += g.size) {
    int ux = (u % nux) * 4, uy = (u / nux) * 4;
    if (usub > 1 && (((uy >> 2) + (ux >> 2)) & 1)) continue;
    int d[16];
    pred::inter_unit4(&ip, uy, ux, d);
    for (int r = 0; r < 4; r++)
      for (int c = 0; c < 4; c++) d[r * 4 + c] = (int)sp[(uy + r) * stride + ux + c] - d[r * 4 + c];
    s += pred::satd4x4(d);
    WORK(W_ANA_SATD, 1);
    WORK(W_ANA_INTER_PX, 16);
  }
  return gsum(s, g) * usub;
}

// LAST, second reference and compound-average SATDs of all planes with each
// plane's two predictions computed once (inter3_satd, k_analysis.h:202-235).
__device__ void inter3(const FrameParams *fp, const uint8_t *src, const uint8_t *ref, const uint8_t *ref2, int x, int y,
                       int w, int h, int mvr, int mvc, int mvr2, int mvc2, long long *s, const Grp &g) {
  long long a0 = 0, a1 = 0, a2 = 0;
  for (int p = 0; p < 3; p++) {
    int sub = p > 0;
    int bx = x >> sub, by = y >> sub, bw = w >> sub, bh = h >> sub, stride = fp->stride[p];
    pred::Inter pa, pb;
    pred::inter_setup(&pa, ref + fp->offset[p], stride, fp->frame_w, fp->frame_h, bx, by, bw, bh, mvr, mvc, sub, sub,
                      EIGHTTAP);
    pred::inter_setup(&pb, ref2 + fp->offset[p], stride, fp->frame_w, fp->frame_h, bx, by, bw, bh, mvr2, mvc2, sub,
                      sub, EIGHTTAP);
    const uint8_t *sp = src + fp->offset[p] + by * stride + bx;
    int usub = eval_sub(fp) && bw >= 32 ? 2 : 1;
    int nux = bw >> 2, nu = nux * (bh >> 2);
    int l0 = 0, l1 = 0, l2 = 0;
    for (int u = g.rank; u < nu; u += g.size) {
      int ux = (u % nux) * 4, uy = (u / nux) * 4;
      if (usub > 1 && (((uy >> 2) + (ux >> 2)) & 1)) continue;
      int d0[16], d1[16], d2[16];
      pred::inter_unit4(&pa, uy, ux, d0);
      pred::inter_unit4(&pb, uy, ux, d1);
      for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) {
          int sv = sp[(uy + r) * stride + ux + c];
          int va = d0[r * 4 + c], vb = d1[r * 4 + c];
          d0[r * 4 + c] = sv - va;
          d1[r * 4 + c] = sv - vb;
          d2[r * 4 + c] = sv - ((va + vb + 1) >> 1);
        }
      l0 += pred::satd4x4(d0);
      l1 += pred::satd4x4(d1);
      l2 += pred::satd4x4(d2);
      WORK(W_ANA_SATD, 3);
      WORK(W_ANA_INTER_PX, 32);
    }
    a0 += (long long)l0 * usub;
    a1 += (long long)l1 * usub;
    a2 += (long long)l2 * usub;
  }
  s[0] = gsum64(a0, g);
  s[1] = gsum64(a1, g);
  s[2] = gsum64(a2, g);
}

// ---- intra SATDs ----------------------------------------------------------------

// Prediction arguments of the analysis (source neighbours, no edge filter,
// no above-right / below-left; intra_satd, k_analysis.h:126-144).
__device__ __forceinline__ pred::IntraArgs ana_args(const FrameParams *fp, int planeIdx, int x, int y, int lw, int lh,
                                                    int mode, int delta) {
  pred::IntraArgs a;
  int sub = planeIdx > 0;
  a.haveLeft = x > 0;
  a.haveAbove = y > 0;
  a.haveAboveRight = 0;
  a.haveBelowLeft = 0;
  a.mode = mode;
  a.angleDelta = delta;
  a.log2W = lw;
  a.log2H = lh;
  a.maxX = ((fp->mi_cols * 4) >> sub) - 1;
  a.maxY = ((fp->mi_rows * 4) >> sub) - 1;
  a.edgeFilter = 0;
  a.filterType = 0;
  return a;
}

// Edge arrays of one plane block (mode independent without the edge filter).
__device__ void build_edges(const FrameParams *fp, const uint8_t *plane, int stride, int planeIdx, int x, int y, int lw,
                            int lh, int *above, int *left, const Grp &g) {
  pred::IntraArgs a = ana_args(fp, planeIdx, x, y, lw, lh, DC_PRED, 0);
  int n = (1 << lw) + (1 << lh);
  for (int i = g.rank; i < n; i += g.size) {
    above[i] = pred::above_sample(plane, stride, x, y, a, i);
    left[i] = pred::left_sample(plane, stride, x, y, a, i);
  }
  if (g.rank == 0) above[-1] = left[-1] = pred::corner_sample(plane, stride, x, y, a);
  gsync(g);
}

// block_satd_s of the intra prediction `mode` (+delta) against the source.
__device__ int intra_mode_satd(const FrameParams *fp, const uint8_t *plane, int stride, int planeIdx, int x, int y,
                               int lw, int lh, int mode, int delta, const int *above, const int *left, const Grp &g) {
  pred::IntraArgs a = ana_args(fp, planeIdx, x, y, lw, lh, mode, delta);
  pred::IntraState st;
  pred::intra_state(a, &st);
  int dc = mode == DC_PRED ? pred::intra_dc(a, above, left) : 0;
  int w = 1 << lw, h = 1 << lh, nux = w >> 2, nu = nux * (h >> 2), s = 0;
  const uint8_t *sp = plane + y * stride + x;
  for (int u = g.rank; u < nu; u += g.size) {
    int ux = (u % nux) * 4, uy = (u / nux) * 4;
    int d[16];
    for (int r = 0; r < 4; r++)
      for (int c = 0; c < 4; c++) {
        int pv = mode == DC_PRED ? dc : pred::intra_pixel(a, st, above, left, uy + r, ux + c);
        d[r * 4 + c] = (int)sp[(uy + r) * stride + ux + c] - pv;
      }
    s += pred::satd4x4(d);
    WORK(W_ANA_SATD, 1);
    WORK(W_ANA_INTRA_PX, 16);
  }
  return gsum(s, g);
}

// CfL SATD of one chroma plane from source luma: DC prediction, the first
// minimum-SSE alpha in [-16, 16], then the SATD of the CfL prediction
// (k_analysis.h:349-365 with cfl_best_alpha / cfl_predict, k_intra.h:252-313).
__device__ int cfl_plane_satd(const FrameParams *fp, const uint8_t *src, int p, int cx, int cy, int clw, int clh,
                              int maxLumaW, int maxLumaH, const int *above, const int *left, const Grp &g) {
  pred::IntraArgs a = ana_args(fp, p, cx, cy, clw, clh, DC_PRED, 0);
  int dc = pred::intra_dc(a, above, left);
  int cw = 1 << clw, ch = 1 << clh, n = cw * ch;
  const uint8_t *luma = src + fp->offset[0];
  int ls = fp->stride[0], stride = fp->stride[p];
  const uint8_t *sp = src + fp->offset[p] + cy * stride + cx;
  int sum = 0;
  for (int k = g.rank; k < n; k += g.size) sum += pred::cfl_luma(luma, ls, cx, cy, maxLumaW, maxLumaH, k / cw, k % cw);
  int avg = round2(gsum(sum, g), clw + clh);
  int sse[33];
  for (int al = 0; al < 33; al++) sse[al] = 0;
  if (g.rank == 0) WORK(W_ANA_CFL, n * 33);
  for (int k = g.rank; k < n; k += g.size) {
    int i = k / cw, j = k % cw;
    int v = pred::cfl_luma(luma, ls, cx, cy, maxLumaW, maxLumaH, i, j) - avg;
    int s0 = sp[i * stride + j];
    for (int al = 0; al < 33; al++) {
      int d = clip3(0, 255, dc + round2signed((al - 16) * v, 6)) - s0;
      sse[al] += d * d;
    }
  }
  int bestA = 0;
  long long best = -1;
  for (int al = 0; al < 33; al++) {
    long long t = gsum64(sse[al], g);
    if (best < 0 || t < best) {
      best = t;
      bestA = al - 16;
    }
  }
  int nux = cw >> 2, nu = nux * (ch >> 2), s = 0;
  for (int u = g.rank; u < nu; u += g.size) {
    int ux = (u % nux) * 4, uy = (u / nux) * 4;
    int d[16];
    for (int r = 0; r < 4; r++)
      for (int c = 0; c < 4; c++) {
        int v = pred::cfl_luma(luma, ls, cx, cy, maxLumaW, maxLumaH, uy + r, ux + c);
        d[r * 4 + c] = (int)sp[(uy + r) * stride + ux + c] - pred::cfl_pixel(dc, bestA, v, avg);
      }
    s += pred::satd4x4(d);
    WORK(W_ANA_SATD, 1);
    WORK(W_ANA_INTRA_PX, 16);
  }
  return gsum(s, g);
}

// ---- eval_block (k_analysis.h:241-404) --------------------------------------------
__device__ long long eval_block(const Ctx &c, int mvNode, int miRow, int miCol, int bsize, BlockInfo *out,
                                WarpMem &wm, const Grp &g) {
  const FrameParams *fp = c.fp;
  int lw = T(Mi_Width_Log2)[bsize] + 2, lh = T(Mi_Height_Log2)[bsize] + 2;
  int w = 1 << lw, h = 1 << lh;
  int x = miCol * 4, y = miRow * 4;
  int lam = fp->ac_q[0] / 16;
  int cx = x >> 1, cy = y >> 1, clw = lw - 1, clh = lh - 1;
  long long interCost = -1;
  int mvr = 0, mvc = 0, refFrame = LAST_FRAME, refFrame1 = 0, mvr1 = 0, mvc1 = 0;
  int sbIdx = (y >> 6) * fp->sb_cols + (x >> 6);
  if (!fp->frame_is_intra && fp->golden && fp->compound) {
    const int32_t *m0 = c.mv + (sbIdx * NUM_NODES + mvNode) * 2;
    const int32_t *m1 = c.mvg + (sbIdx * NUM_NODES + mvNode) * 2;
    int lr = m0[0], lc = m0[1], gr = m1[0], gc = m1[1];
    long long s[3];
    inter3(fp, c.src, c.ref, c.gold, x, y, w, h, lr, lc, gr, gc, s, g);
    interCost = s[0] + (long long)lam * (4 + mv_bits8(lr, lc)) / 8;
    mvr = lr;
    mvc = lc;
    long long g = s[1] + (long long)lam * (4 + mv_bits8(gr, gc)) / 8 + (long long)lam * GOLDEN_REF_BITS8 / 8;
    if (g < interCost) {
      interCost = g;
      mvr = gr;
      mvc = gc;
      refFrame = fp->ref2_frame;
    }
    long long cc = s[2] + (long long)lam * (8 + mv_bits8(lr, lc) + mv_bits8(gr, gc) + COMPOUND_BITS8) / 8;
    if (cc < interCost) {
      interCost = cc;
      mvr = lr;
      mvc = lc;
      mvr1 = gr;
      mvc1 = gc;
      refFrame = LAST_FRAME;
      refFrame1 = fp->ref2_frame;
    }
  } else if (!fp->frame_is_intra) {
    for (int r = 0; r < (fp->golden ? 2 : 1); r++) {
      const int32_t *mp = (r ? c.mvg : c.mv) + (sbIdx * NUM_NODES + mvNode) * 2;
      const uint8_t *rp = r ? c.gold : c.ref;
      int qr = mp[0], qc = mp[1];
      long long cost = inter_plane_satd(fp, c.src, rp, 0, x, y, w, h, qr, qc, g);
      for (int p = 1; p < 3; p++) cost += inter_plane_satd(fp, c.src, rp, p, cx, cy, w >> 1, h >> 1, qr, qc, g);
      cost += (long long)lam * (4 + mv_bits8(qr, qc)) / 8;
      if (r == 0) {
        interCost = cost;
        mvr = qr;
        mvc = qc;
      } else {
        cost += (long long)lam * GOLDEN_REF_BITS8 / 8;
        if (cost < interCost) { /* tie: LAST */
          interCost = cost;
          mvr = qr;
          mvc = qc;
          refFrame = fp->ref2_frame;
        }
      }
    }
  }
  // luma intra
  long long best = -1;
  int bestMode = DC_PRED, bestDelta = 0;
  int skipIntra = interCost >= 0 && (fp->leaf || (fp->fast && interCost * 16 < (long long)w * h * lam * 16));
  int *ya = wm.edge[0][0] + EDGE_OFF, *yl = wm.edge[0][1] + EDGE_OFF;
  if (!skipIntra) {
    build_edges(fp, c.src + fp->offset[0], fp->stride[0], 0, x, y, lw, lh, ya, yl, g);
    for (int mode = DC_PRED; mode <= PAETH_PRED; mode++) {
      if (turbo_mode_off(fp, mode)) continue;
      long long cst = intra_mode_satd(fp, c.src + fp->offset[0], fp->stride[0], 0, x, y, lw, lh, mode, 0, ya, yl, g) +
                      (long long)lam * mode_bits8(mode) / 8;
      if (best < 0 || cst < best) {
        best = cst;
        bestMode = mode;
      }
    }
  }
  if (skipIntra) best = 1LL << 40;
  if (intra_is_directional(bestMode) && !fp->fast) {
    int base = bestMode;
    for (int d = -MAX_ANGLE_DELTA; d <= MAX_ANGLE_DELTA; d++) {
      if (d == 0) continue;
      long long cst = intra_mode_satd(fp, c.src + fp->offset[0], fp->stride[0], 0, x, y, lw, lh, base, d, ya, yl, g) +
                      (long long)lam * (mode_bits8(base) + 16) / 8;
      if (cst < best) {
        best = cst;
        bestDelta = d;
      }
    }
  }
  int skipUv = fp->fast && interCost >= 0 && best + (long long)lam * 16 / 8 >= interCost;
  long long bestUv = skipUv ? 0 : -1;
  int bestUvMode = DC_PRED;
  if (!skipUv) {
    for (int p = 1; p < 3; p++)
      build_edges(fp, c.src + fp->offset[p], fp->stride[p], p, cx, cy, clw, clh, wm.edge[p][0] + EDGE_OFF,
                  wm.edge[p][1] + EDGE_OFF, g);
    for (int m = DC_PRED; m <= PAETH_PRED; m++) {
      if (intra_is_directional(m) && m != V_PRED && m != H_PRED && m != bestMode) continue;
      if (turbo_mode_off(fp, m)) continue;
      int delta = (m == bestMode) ? bestDelta : 0;
      long long cst = 0;
      for (int p = 1; p < 3; p++)
        cst += intra_mode_satd(fp, c.src + fp->offset[p], fp->stride[p], p, cx, cy, clw, clh, m, delta,
                               wm.edge[p][0] + EDGE_OFF, wm.edge[p][1] + EDGE_OFF, g);
      cst += (long long)lam * (m == DC_PRED ? 8 : 24) / 8;
      if (bestUv < 0 || cst < bestUv) {
        bestUv = cst;
        bestUvMode = m;
      }
    }
    if (cfl_allowed(bsize, fp->lossless) && !turbo_no_cfl(fp)) {
      long long cst = (long long)lam * 40 / 8;
      for (int p = 1; p < 3; p++)
        cst += cfl_plane_satd(fp, c.src, p, cx, cy, clw, clh, x + w, y + h, wm.edge[p][0] + EDGE_OFF,
                              wm.edge[p][1] + EDGE_OFF, g);
      if (cst < bestUv) {
        bestUv = cst;
        bestUvMode = UV_CFL_PRED;
      }
    }
  }
  BlockInfo b;
  b.mi_row = miRow;
  b.mi_col = miCol;
  b.bsize = bsize;
  b.is_inter = 0;
  b.y_mode = bestMode;
  b.angle_y = bestDelta;
  b.uv_mode = bestUvMode;
  b.angle_uv = (bestUvMode == bestMode) ? bestDelta : 0;
  b.cfl_alpha_u = b.cfl_alpha_v = 0;
  b.tx_depth = 0;
  b.interp_filter = 0;
  b.tx_types_lo = b.tx_types_hi = 0;
  b.mv_row = b.mv_col = 0;
  b.ref_frame = INTRA_FRAME;
  b.ref_frame1 = 0;
  b.mv1_row = b.mv1_col = 0;
  b.tx_type = DCT_DCT;
  b.eob[0] = b.eob[1] = b.eob[2] = 0;
  b.coef_off[0] = b.coef_off[1] = b.coef_off[2] = 0;
  long long cost = best + bestUv + (long long)lam * (fp->frame_is_intra ? 0 : 16) / 8;
  if (interCost >= 0 && interCost < cost) {
    cost = interCost;
    b.is_inter = 1;
    b.y_mode = NEWMV;
    b.uv_mode = DC_PRED;
    b.angle_y = 0;
    b.angle_uv = 0;
    b.mv_row = mvr;
    b.mv_col = mvc;
    b.ref_frame = refFrame;
    b.ref_frame1 = refFrame1;
    b.mv1_row = mvr1;
    b.mv1_col = mvc1;
  }
  *out = b;
  return cost;
}

// ---- partition geometry (k_analysis.h:408-443, 590-631, 682-694) ------------------
HD int part_block(int p, int bSize, int k, int halfMi, int *dr, int *dc) {
  int sub = T(Partition_Subsize)[p][bSize], split = T(Partition_Subsize)[PARTITION_SPLIT][bSize];
  int q = halfMi >> 1;
  *dr = 0;
  *dc = 0;
  switch (p) {
    case PARTITION_HORZ: *dr = k * halfMi; return sub;
    case PARTITION_VERT: *dc = k * halfMi; return sub;
    case PARTITION_HORZ_A:
      if (k < 2) { *dc = k * halfMi; return split; }
      *dr = halfMi; return sub;
    case PARTITION_HORZ_B:
      if (k == 0) return sub;
      *dr = halfMi; *dc = (k - 1) * halfMi; return split;
    case PARTITION_VERT_A:
      if (k < 2) { *dr = k * halfMi; return split; }
      *dc = halfMi; return sub;
    case PARTITION_VERT_B:
      if (k == 0) return sub;
      *dc = halfMi; *dr = (k - 1) * halfMi; return split;
    case PARTITION_HORZ_4: *dr = k * q; return sub;
    case PARTITION_VERT_4: *dc = k * q; return sub;
    default: return sub;
  }
}

HD int part_count(const FrameParams *fp, int p, int r, int c, int halfMi) {
  int hasRows = (r + halfMi) < fp->mi_rows, hasCols = (c + halfMi) < fp->mi_cols;
  if (p == PARTITION_NONE) return 1;
  if (p == PARTITION_HORZ) return hasRows ? 2 : 1;
  if (p == PARTITION_VERT) return hasCols ? 2 : 1;
  if (p == PARTITION_HORZ_4) return (r + (halfMi >> 1) * 3 < fp->mi_rows) ? 4 : 3;
  if (p == PARTITION_VERT_4) return (c + (halfMi >> 1) * 3 < fp->mi_cols) ? 4 : 3;
  return 3;
}

HD void slot_part(int slot, int *p, int *k) {
  if (slot == 0) { *p = PARTITION_NONE; *k = 0; }
  else if (slot < 3) { *p = PARTITION_HORZ; *k = slot - 1; }
  else if (slot < 5) { *p = PARTITION_VERT; *k = slot - 3; }
  else if (slot < 9) { *p = PARTITION_HORZ_4; *k = slot - 5; }
  else { *p = PARTITION_VERT_4; *k = slot - 9; }
}

HD int turbo_square(const FrameParams *fp) {
  return (fp->turbo & T_SQUARE) && (!fp->frame_is_intra || (fp->turbo & T_KEY_SQUARE));
}
HD int leaf_no8(const FrameParams *fp) { return (fp->turbo & T_LEAF_NO8) && fp->leaf && !fp->frame_is_intra; }
HD int node8_at_edge(const FrameParams *fp, int sbIdx, int i) {
  int r = (sbIdx / fp->sb_cols) * 16 + ((i >> 3) & ~1) * 2, c = (sbIdx % fp->sb_cols) * 16 + ((i & 7) & ~1) * 2;
  return r + 4 > fp->mi_rows || c + 4 > fp->mi_cols;
}

HD int part_allowed(const FrameParams *fp, int level, int p, int hasRows, int hasCols) {
  if (p == PARTITION_SPLIT) return 0;
  if (level == 3 && p != PARTITION_NONE) return 0;
  if (fp->fast && p > PARTITION_SPLIT) return 0;
  if (turbo_square(fp) && p != PARTITION_NONE) return 0;
  if (level == 2 && (p == PARTITION_HORZ_4 || p == PARTITION_VERT_4)) return 0;
  if (!(hasRows && hasCols))
    return (p == PARTITION_HORZ && hasCols && !hasRows) || (p == PARTITION_VERT && hasRows && !hasCols);
  return 1;
}

HD int level_slots(const FrameParams *fp, int level) {
  if (level == 3 || turbo_square(fp)) return 1;
  if (level == 2 || fp->fast) return 5;
  return A_SLOTS;
}

HD int part_slot(int p, int k) {
  switch (p) {
    case PARTITION_NONE: return 0;
    case PARTITION_HORZ: return 1 + k;
    case PARTITION_VERT: return 3 + k;
    case PARTITION_HORZ_4: return 5 + k;
    case PARTITION_VERT_4: return 9 + k;
    case PARTITION_HORZ_A: return k < 2 ? -1 : 2;
    case PARTITION_HORZ_B: return k == 0 ? 1 : -1;
    case PARTITION_VERT_A: return k < 2 ? -1 : 4;
    default: return k == 0 ? 3 : -1;
  }
}

// Depth early exit (k_analysis.h:642-654).
__device__ int depth_pruned(const FrameParams *fp, const int64_t *costs, int sbIdx, int level, int i) {
  if (!fp->fast || level == 0 || fp->depth_thr == 0) return 0;
  int y = i >> level, x = i & ((1 << level) - 1);
  for (int a = level - 1; a >= 0; a--) {
    y >>= 1;
    x >>= 1;
    long long pc = costs[(long long)sbIdx * A_ITEMS + (node_base(a) + (y << a) + x) * A_SLOTS];
    int pw = 64 >> a;
    if (pc >= 0 && pc * 16 < (long long)pw * pw * fp->depth_thr) return 1;
  }
  return 0;
}

// Pass 1 of one level: items (superblock, node, slot) in the reference's
// order sb-major (k_analysis.h:656-679). A warp per item, or with
// whole_cta the CTA's four warps on one item (the 64x64 level, whose few
// large items would otherwise leave most SMs idle).
#define ANA_THREADS 128
// group: threads per candidate (ANA_THREADS, 32 or 16; ana_groups gives the
// edge scratch areas the dynamic shared memory holds).
__host__ __device__ constexpr int ana_groups(int group) { return group < 32 ? ANA_THREADS / group : ANA_THREADS / 32; }
// At least 4 CTAs per SM (at most 128 registers a thread): the level's
// candidates are latency-bound SATD and filter sums, and the extra resident
// warps hide more of it (measured on the 1080p clip: key-frame analysis
// 2.47 -> 1.74 ms at 168 -> 128 registers; 5 CTAs spill and lose again).
#ifndef MAV1CU_ANA_MIN_CTAS
#define MAV1CU_ANA_MIN_CTAS 4
#endif
__global__ void __launch_bounds__(ANA_THREADS, MAV1CU_ANA_MIN_CTAS) k_analyze_level(Ctx c, int level, int slots, int group) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WarpMem *wmem = (WarpMem *)smem_raw;
  long long *red = (long long *)(wmem + ana_groups(group));
  const FrameParams *fp = c.fp;
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, half = lane >> 4;
  int whole_cta = group == ANA_THREADS;
  int gi = whole_cta ? 0 : group == 32 ? warp : 2 * warp + half;
  int n = 1 << level, per = n * n * slots;
  int item = whole_cta ? (int)blockIdx.x : (int)blockIdx.x * (ANA_THREADS / group) + gi;
  Grp grp = whole_cta ? Grp{(int)threadIdx.x, ANA_THREADS, red, 0xffffffffu}
            : group == 32 ? Grp{lane, 32, nullptr, 0xffffffffu}
                          : Grp{lane & 15, 16, nullptr, 0xffffu << (16 * half)};
  WarpMem &wm = wmem[gi];
  if (item >= fp->sb_cols * fp->sb_rows * per) return;
  int sbIdx = item / per, rem = item % per, i = rem / slots, slot = rem % slots;
  int sbRow = sbIdx / fp->sb_cols, sbCol = sbIdx % fp->sb_cols;
  int size4 = 16 >> level, halfSz = size4 >> 1;
  int node = node_base(level) + i;
  int r = sbRow * 16 + (i / n) * size4, cc = sbCol * 16 + (i % n) * size4;
  long long idx = (long long)sbIdx * A_ITEMS + node * A_SLOTS + slot;
  bool skip = r >= fp->mi_rows || cc >= fp->mi_cols || depth_pruned(fp, c.costs, sbIdx, level, i) ||
              (level == 3 && leaf_no8(fp) && !node8_at_edge(fp, sbIdx, i));
  int p = 0, k = 0, hasRows = 0, hasCols = 0;
  if (!skip) {
    hasRows = (r + halfSz) < fp->mi_rows;
    hasCols = (cc + halfSz) < fp->mi_cols;
    slot_part(slot, &p, &k);
    skip = !part_allowed(fp, level, p, hasRows, hasCols) || k >= part_count(fp, p, r, cc, halfSz);
  }
  if (skip) {
    if (grp.rank == 0) c.costs[idx] = -1;
    return;
  }
  int dr, dc;
  int bs = part_block(p, level_bsize(level), k, halfSz, &dr, &dc);
  BlockInfo b;
  long long cost = eval_block(c, node, r + dr, cc + dc, bs, &b, wm, grp);
  if (grp.rank == 0) {
    c.costs[idx] = cost;
    c.infos[idx] = b;
  }
}

// Pass 2: partition decision and block emission (k_analysis.h:697-808), one
// warp per superblock. The nodes of a level are independent: lanes take
// them, bottom-up level by level, with the costs in shared memory. Emission
// walks the 64 8x8 positions in Z order: each lane finds the blocks its
// positions emit, a warp prefix sum of their counts and coefficient sizes
// gives every block its index and coefficient offsets (the serial walk's).
#define TABLE_WARPS 4
struct TableMem {
  long long cost[NUM_NODES], noneCost[NUM_NODES];
  int part[NUM_NODES];
};

__device__ __forceinline__ int warp_excl_scan(int v, int lane, int *total) {
  int x = v;
  for (int off = 1; off < 32; off <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, off);
    if (lane >= off) x += y;
  }
  *total = __shfl_sync(0xffffffffu, x, 31);
  return x - v;
}

__global__ void __launch_bounds__(32 * TABLE_WARPS) k_analyze_table(Ctx c) {
  __shared__ TableMem tms[TABLE_WARPS];
  const FrameParams *fp = c.fp;
  int lane = threadIdx.x & 31, sbIdx = blockIdx.x * TABLE_WARPS + (threadIdx.x >> 5);
  if (sbIdx >= fp->sb_cols * fp->sb_rows) return;
  TableMem &m = tms[threadIdx.x >> 5];
  int sbRow = sbIdx / fp->sb_cols, sbCol = sbIdx % fp->sb_cols;
  int lam = fp->ac_q[0] / 16;
  const int64_t *tc = c.costs + (long long)sbIdx * A_ITEMS;
  const BlockInfo *ti = c.infos + (long long)sbIdx * A_ITEMS;
  for (int level = 3; level >= 0; level--) {
    int n = 1 << level, size4 = 16 >> level, bSize = level_bsize(level);
    for (int i = lane; i < n * n; i += 32) {
      int node = node_base(level) + i;
      int r = sbRow * 16 + (i / n) * size4, cc = sbCol * 16 + (i % n) * size4;
      m.noneCost[node] = -1;
      if (r >= fp->mi_rows || cc >= fp->mi_cols) {
        m.cost[node] = 0;
        m.part[node] = -1;
        continue;
      }
      int halfSz = size4 >> 1;
      int hasRows = (r + halfSz) < fp->mi_rows, hasCols = (cc + halfSz) < fp->mi_cols;
      int cn = n * 2, ci = (i / n) * 2 * cn + (i % n) * 2, cb = level < 3 ? node_base(level + 1) : 0;
      long long bestC = -1;
      int bestP = PARTITION_SPLIT;
      if (level < 3) {
        long long c0 = m.cost[cb + ci], c1 = m.cost[cb + ci + 1], c2 = m.cost[cb + ci + cn], c3 = m.cost[cb + ci + cn + 1];
        if (c0 >= 0 && c1 >= 0 && c2 >= 0 && c3 >= 0) bestC = c0 + c1 + c2 + c3 + (long long)lam * 16 / 8;
      }
      long long noneC = -1;
      for (int p = PARTITION_NONE; p <= PARTITION_VERT_4; p++) {
        if (!part_allowed(fp, level, p, hasRows, hasCols)) continue;
        long long pc = 0;
        int nb = part_count(fp, p, r, cc, halfSz);
        for (int k = 0; k < nb && pc >= 0; k++) {
          int s = part_slot(p, k);
          long long v;
          if (s < 0) {
            int dr, dc;
            part_block(p, bSize, k, halfSz, &dr, &dc);
            v = m.noneCost[cb + ci + (dr ? cn : 0) + (dc ? 1 : 0)];
          } else {
            v = tc[node * A_SLOTS + s];
          }
          pc = v < 0 ? -1 : pc + v;
        }
        if (pc < 0) continue;
        pc += (long long)lam * (p == PARTITION_NONE ? 8 : 24) / 8;
        if (p == PARTITION_NONE) noneC = pc;
        if (bestC < 0 || pc <= bestC) {
          bestC = pc;
          bestP = p;
        }
      }
      m.noneCost[node] = noneC;
      m.cost[node] = bestC;
      m.part[node] = bestP;
    }
    __syncwarp();
  }
  SbInfo *sb = &c.sbs[sbIdx];
  for (int k = lane; k < NUM_NODES; k += 32) sb->part[k] = m.part[k];
  // the blocks each of this lane's two Z positions emits
  int nbz[2], nodez[2], levz[2], zyz[2], zxz[2], coefz[2];
  for (int h = 0; h < 2; h++) {
    int z = lane + 32 * h, zx = 0, zy = 0;
    for (int bb = 0; bb < 3; bb++) {
      zx |= ((z >> (2 * bb)) & 1) << bb;
      zy |= ((z >> (2 * bb + 1)) & 1) << bb;
    }
    nbz[h] = 0;
    coefz[h] = 0;
    zxz[h] = zx;
    zyz[h] = zy;
    for (int level = 0; level <= 3; level++) {
      int shift = 3 - level, n = 1 << level;
      int node = node_base(level) + (zy >> shift) * n + (zx >> shift);
      int p = m.part[node];
      if (p < 0) break;
      if (p == PARTITION_SPLIT) continue;
      if ((zx & ((1 << shift) - 1)) == 0 && (zy & ((1 << shift) - 1)) == 0) {
        int size4 = 16 >> level, halfMi = size4 >> 1;
        int r = sbRow * 16 + (zy >> shift) * size4, cc = sbCol * 16 + (zx >> shift) * size4;
        nbz[h] = part_count(fp, p, r, cc, halfMi);
        nodez[h] = node;
        levz[h] = level;
        int cn = n * 2, ci = (zy >> shift) * 2 * cn + (zx >> shift) * 2, cb = level < 3 ? node_base(level + 1) : 0;
        for (int k = 0; k < nbz[h]; k++) {
          int s = part_slot(p, k), bsz;
          if (s < 0) {
            int dr, dc;
            part_block(p, level_bsize(level), k, halfMi, &dr, &dc);
            bsz = ti[(cb + ci + (dr ? cn : 0) + (dc ? 1 : 0)) * A_SLOTS].bsize;
          } else {
            bsz = ti[node * A_SLOTS + s].bsize;
          }
          int w = block_w(bsz), hh = block_h(bsz);
          coefz[h] += w * hh + 2 * ((w >> 1) * (hh >> 1));
        }
      }
      break;
    }
  }
  int t0, t1, c0t, c1t;
  int base0 = warp_excl_scan(nbz[0], lane, &t0), base1 = t0 + warp_excl_scan(nbz[1], lane, &t1);
  int cbase0 = warp_excl_scan(coefz[0], lane, &c0t), cbase1 = c0t + warp_excl_scan(coefz[1], lane, &c1t);
  for (int h = 0; h < 2; h++) {
    int count = h ? base1 : base0, coefOff = sbIdx * COEFS_PER_SB + (h ? cbase1 : cbase0);
    if (!nbz[h]) continue;
    int level = levz[h], node = nodez[h], shift = 3 - level, n = 1 << level, p = m.part[node];
    int zx = zxz[h], zy = zyz[h], halfMi = (16 >> level) >> 1;
    int cn = n * 2, ci = (zy >> shift) * 2 * cn + (zx >> shift) * 2, cb = level < 3 ? node_base(level + 1) : 0;
    for (int k = 0; k < nbz[h]; k++) {
      int s = part_slot(p, k);
      BlockInfo b;
      if (s < 0) {
        int dr, dc;
        part_block(p, level_bsize(level), k, halfMi, &dr, &dc);
        b = ti[(cb + ci + (dr ? cn : 0) + (dc ? 1 : 0)) * A_SLOTS];
      } else {
        b = ti[node * A_SLOTS + s];
      }
      int w = block_w(b.bsize), hh = block_h(b.bsize);
      b.coef_off[0] = coefOff;
      coefOff += w * hh;
      b.coef_off[1] = coefOff;
      coefOff += (w >> 1) * (hh >> 1);
      b.coef_off[2] = coefOff;
      coefOff += (w >> 1) * (hh >> 1);
      b.eob[0] = b.eob[1] = b.eob[2] = 0;
      c.blocks[sbIdx * MAX_BLOCKS_PER_SB + count] = b;
      count++;
    }
  }
  if (lane == 0) {
    sb->first_block = sbIdx * MAX_BLOCKS_PER_SB;
    sb->num_blocks = t0 + t1;
    sb->sb_row = sbRow;
    sb->sb_col = sbCol;
  }
}

// ---- intra edge filter types (encoder.c:319-346) ------------------------------------
HD int smooth_mode(int m) { return m == SMOOTH_PRED || m == SMOOTH_V_PRED || m == SMOOTH_H_PRED; }

// Step 1: every mi covered by a block gets its luma / chroma smooth flag.
__global__ void k_edge_marks(const FrameParams *fp, const BlockInfo *blocks, const SbInfo *sbs, uint8_t *ys,
                             uint8_t *uvs) {
  int sb = blockIdx.x, k = threadIdx.x;
  if (k >= sbs[sb].num_blocks) return;
  const BlockInfo *b = &blocks[sbs[sb].first_block + k];
  int cols = fp->mi_cols, rows = fp->mi_rows;
  int ysm = smooth_mode(b->y_mode) && !b->is_inter, uvsm = !b->is_inter && smooth_mode(b->uv_mode);
  for (int r = b->mi_row; r < b->mi_row + T(Num_4x4_Blocks_High)[b->bsize] && r < rows; r++)
    for (int cc = b->mi_col; cc < b->mi_col + T(Num_4x4_Blocks_Wide)[b->bsize] && cc < cols; cc++) {
      ys[r * cols + cc] = (uint8_t)ysm;
      uvs[r * cols + cc] = (uint8_t)uvsm;
    }
}

// Step 2: get_filter_type( ) of each block from its above / left neighbours.
__global__ void k_edge_types(const FrameParams *fp, BlockInfo *blocks, const SbInfo *sbs, const uint8_t *ys,
                             const uint8_t *uvs) {
  int sb = blockIdx.x, k = threadIdx.x;
  if (k >= sbs[sb].num_blocks) return;
  BlockInfo *b = &blocks[sbs[sb].first_block + k];
  int cols = fp->mi_cols, rows = fp->mi_rows;
  int r = b->mi_row, cc = b->mi_col;
  int availU = r > 0, availL = cc > tile_col_start(fp, cc);
  int fy = (availU && ys[(r - 1) * cols + cc]) || (availL && ys[r * cols + cc - 1]);
  int fuv = (availU && uvs[(r - 1) * cols + imin(cc + 1, cols - 1)]) || (availL && uvs[imin(r + 1, rows - 1) * cols + cc - 1]);
  b->interp_filter = (b->interp_filter & 15) | fy << 4 | fuv << 5;
}

}  // namespace ana
