// Inter and intra prediction, per output sample.
//
// Inter: translational prediction from an unscaled reference (AV1 spec
// 7.11.3.3-7.11.3.4 with xScale = yScale = 1 << 14). With an unscaled
// reference the spec's position arithmetic reduces exactly to
//   P = (x << 4) + ((2 * mv) >> sub),  integer sample P >> 4,  phase P & 15
// (startX = 64 * P + 32 and every step is 1024), so each output sample is the
// 8-tap vertical filter (Round2 by InterRound1) of eight 8-tap horizontal
// intermediates (Round2 by InterRound0 = 3) of clamped reference samples,
// the same values the reference's predict_inter_block produces
// (src/kernels/k_inter.h:451-504, 510-563). A thread computes whole samples;
// nothing is staged, so any thread can predict any sample.
//
// Intra: spec 7.11.2. The edge arrays (AboveRow / LeftCol, with the edge
// filter and upsampling of directional modes) are built cooperatively in
// shared memory by a thread group, then every sample is predicted
// independently (reference src/kernels/k_intra.h:92-248).
#pragma once

#include "common.cuh"

namespace pred {

// ---- inter -------------------------------------------------------------------
struct Inter {
  const uint8_t *ref;  // plane origin
  int stride, lastX, lastY;
  int ix0, iy0;        // integer position of output sample (0, 0) minus 3
  int fullpel;         // both filter positions 0: every filter is the identity there
  int16_t fh[8], fv[8];  // taps span -128..128
};

// filter: InterpFilters[0] (vertical) | InterpFilters[1] (horizontal) << 2.
HD void inter_setup(Inter *p, const uint8_t *ref, int stride, int refW, int refH, int x, int y, int w, int h, int mvRow,
                    int mvCol, int subX, int subY, int filter) {
  int px = (x << 4) + ((2 * mvCol) >> subX);
  int py = (y << 4) + ((2 * mvRow) >> subY);
  p->ref = ref;
  p->stride = stride;
  p->lastX = ((refW + subX) >> subX) - 1;
  p->lastY = ((refH + subY) >> subY) - 1;
  p->ix0 = (px >> 4) - 3;
  p->iy0 = (py >> 4) - 3;
  p->fullpel = ((px | py) & 15) == 0;
  int fv = filter & 3, fh = (filter >> 2) & 3;
  if (w <= 4) fh = (fh == EIGHTTAP || fh == EIGHTTAP_SHARP) ? 4 : (fh == EIGHTTAP_SMOOTH ? 5 : fh);
  if (h <= 4) fv = (fv == EIGHTTAP || fv == EIGHTTAP_SHARP) ? 4 : (fv == EIGHTTAP_SMOOTH ? 5 : fv);
  const int32_t *FH = T(Subpel_Filters)[fh][px & 15], *FV = T(Subpel_Filters)[fv][py & 15];
  for (int t = 0; t < 8; t++) {
    p->fh[t] = (int16_t)FH[t];
    p->fv[t] = (int16_t)FV[t];
  }
}

// Vertical filter sum of output sample (r, c) before its final rounding.
HD int inter_sum(const Inter *p, int r, int c) {
  int xs[8];
  for (int t = 0; t < 8; t++) xs[t] = clip3(0, p->lastX, p->ix0 + c + t);
  int acc = 0;
  for (int tv = 0; tv < 8; tv++) {
    const uint8_t *row = p->ref + (size_t)clip3(0, p->lastY, p->iy0 + r + tv) * p->stride;
    int s = 0;
    for (int t = 0; t < 8; t++) s += p->fh[t] * (int)row[xs[t]];
    acc += p->fv[tv] * round2(s, 3);
  }
  return acc;
}

// Single-reference sample: Clip1( Round2( sum, 11 ) ).
HD int inter_pixel(const Inter *p, int r, int c) { return clip1(round2(inter_sum(p, r, c), 11)); }
// Compound intermediate (isCompound: InterRound1 = 7, not clipped).
HD int inter_raw(const Inter *p, int r, int c) { return round2(inter_sum(p, r, c), 7); }

// The 16 single-reference samples of the 4x4 unit at (r0, c0), row-major
// into o: inter_pixel in separable form. A horizontal sum Round2( ., 3 )
// depends only on its row and column, so the unit's 11 x 4 of them are
// formed once (11 x 11 reference samples) and each output takes 8 of them;
// at a full-sample position every filter is (0, 0, 0, 128, 0, 0, 0, 0) and
// the prediction is the clamped reference sample itself.
HD void inter_unit4(const Inter *p, int r0, int c0, int *o) {
  if (p->fullpel) {
    for (int r = 0; r < 4; r++) {
      const uint8_t *row = p->ref + (size_t)clip3(0, p->lastY, p->iy0 + 3 + r0 + r) * p->stride;
      for (int c = 0; c < 4; c++) o[r * 4 + c] = row[clip3(0, p->lastX, p->ix0 + 3 + c0 + c)];
    }
    return;
  }
  int xs[11];
  for (int t = 0; t < 11; t++) xs[t] = clip3(0, p->lastX, p->ix0 + c0 + t);
  int hs[11][4];
  for (int tv = 0; tv < 11; tv++) {
    const uint8_t *row = p->ref + (size_t)clip3(0, p->lastY, p->iy0 + r0 + tv) * p->stride;
    int px[11];
    for (int t = 0; t < 11; t++) px[t] = row[xs[t]];
    for (int c = 0; c < 4; c++) {
      int s = 0;
      for (int t = 0; t < 8; t++) s += p->fh[t] * px[c + t];
      hs[tv][c] = round2(s, 3);
    }
  }
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 4; c++) {
      int acc = 0;
      for (int tv = 0; tv < 8; tv++) acc += p->fv[tv] * hs[r + tv][c];
      o[r * 4 + c] = clip1(round2(acc, 11));
    }
}

// ---- SATD --------------------------------------------------------------------
// 4x4 Hadamard SATD of a difference block d[row * 4 + col] (the analysis
// metric of the reference, src/kernels/k_analysis.h:58-73).
HD int satd4x4(const int *d) {
  int t[16];
  for (int i = 0; i < 4; i++) {
    int a0 = d[i * 4 + 0] + d[i * 4 + 1], a1 = d[i * 4 + 0] - d[i * 4 + 1];
    int a2 = d[i * 4 + 2] + d[i * 4 + 3], a3 = d[i * 4 + 2] - d[i * 4 + 3];
    t[i * 4 + 0] = a0 + a2;
    t[i * 4 + 1] = a1 + a3;
    t[i * 4 + 2] = a0 - a2;
    t[i * 4 + 3] = a1 - a3;
  }
  int s = 0;
  for (int j = 0; j < 4; j++) {
    int a0 = t[0 * 4 + j] + t[1 * 4 + j], a1 = t[0 * 4 + j] - t[1 * 4 + j];
    int a2 = t[2 * 4 + j] + t[3 * 4 + j], a3 = t[2 * 4 + j] - t[3 * 4 + j];
    s += iabs(a0 + a2) + iabs(a1 + a3) + iabs(a0 - a2) + iabs(a1 - a3);
  }
  return s;
}

// ---- intra -------------------------------------------------------------------
#define EDGE_OFF 16
#define EDGE_LEN (EDGE_OFF + 129 * 2 + 16)

struct IntraArgs {
  int haveLeft, haveAbove, haveAboveRight, haveBelowLeft;
  int mode, angleDelta, log2W, log2H;
  int maxX, maxY;
  int edgeFilter, filterType;
};

// Derived state of one prediction, computed identically by every thread.
struct IntraState {
  int pAngle, upAbove, upLeft, dx, dy;
};

HD int edge_strength(int w, int h, int filterType, int delta) {
  int d = iabs(delta), blkWh = w + h, strength = 0;
  if (filterType == 0) {
    if (blkWh <= 8) { if (d >= 56) strength = 1; }
    else if (blkWh <= 12) { if (d >= 40) strength = 1; }
    else if (blkWh <= 16) { if (d >= 40) strength = 1; }
    else if (blkWh <= 24) { if (d >= 8) strength = 1; if (d >= 16) strength = 2; if (d >= 32) strength = 3; }
    else if (blkWh <= 32) { strength = 1; if (d >= 4) strength = 2; if (d >= 32) strength = 3; }
    else strength = 3;
  } else {
    if (blkWh <= 8) { if (d >= 40) strength = 1; if (d >= 64) strength = 2; }
    else if (blkWh <= 16) { if (d >= 20) strength = 1; if (d >= 48) strength = 2; }
    else if (blkWh <= 24) { if (d >= 4) strength = 3; }
    else strength = 3;
  }
  return strength;
}

HD int use_upsample(int w, int h, int filterType, int delta) {
  int d = iabs(delta), blkWh = w + h;
  if (d <= 0 || d >= 40) return 0;
  return filterType == 0 ? (blkWh <= 16) : (blkWh <= 8);
}

HD void intra_state(const IntraArgs &a, IntraState *s) {
  int w = 1 << a.log2W, h = 1 << a.log2H;
  s->pAngle = 0;
  s->upAbove = s->upLeft = 0;
  s->dx = s->dy = 0;
  if (!intra_is_directional(a.mode)) return;
  int pAngle = T(Mode_To_Angle)[a.mode] + a.angleDelta * ANGLE_STEP;
  s->pAngle = pAngle;
  if (a.edgeFilter) {
    s->upAbove = use_upsample(w, h, a.filterType, pAngle - 90);
    s->upLeft = use_upsample(w, h, a.filterType, pAngle - 180);
  }
  if (pAngle < 90) s->dx = T(Dr_Intra_Derivative)[pAngle];
  else if (pAngle > 90 && pAngle < 180) s->dx = T(Dr_Intra_Derivative)[180 - pAngle];
  if (pAngle > 90 && pAngle < 180) s->dy = T(Dr_Intra_Derivative)[pAngle - 90];
  else if (pAngle > 180) s->dy = T(Dr_Intra_Derivative)[270 - pAngle];
}

// Edge sample i (0 <= i < w + h) of AboveRow / LeftCol before filtering.
HD int above_sample(const uint8_t *px, int stride, int x, int y, const IntraArgs &a, int i) {
  int w = 1 << a.log2W;
  if (!a.haveAbove && a.haveLeft) return px[y * stride + x - 1];
  if (!a.haveAbove && !a.haveLeft) return (1 << 7) - 1;
  int aboveLimit = imin(a.maxX, x + (a.haveAboveRight ? 2 * w : w) - 1);
  return px[(y - 1) * stride + imin(aboveLimit, x + i)];
}
HD int left_sample(const uint8_t *px, int stride, int x, int y, const IntraArgs &a, int i) {
  int h = 1 << a.log2H;
  if (!a.haveLeft && a.haveAbove) return px[(y - 1) * stride + x];
  if (!a.haveLeft && !a.haveAbove) return (1 << 7) + 1;
  int leftLimit = imin(a.maxY, y + (a.haveBelowLeft ? 2 * h : h) - 1);
  return px[imin(leftLimit, y + i) * stride + x - 1];
}
HD int corner_sample(const uint8_t *px, int stride, int x, int y, const IntraArgs &a) {
  if (a.haveAbove && a.haveLeft) return px[(y - 1) * stride + x - 1];
  if (a.haveAbove) return px[(y - 1) * stride + x];
  if (a.haveLeft) return px[y * stride + x - 1];
  return 1 << 7;
}

// Builds the edge arrays (above / left point at element 0; index -1 is the
// corner, -2 set by upsampling) with `n` threads of rank `rank`; sync() is
// the group's barrier. Spec 7.11.2 steps 1-6 (edge filter 7.11.2.12,
// upsampling 7.11.2.11).
template <class Sync>
__host__ __device__ void intra_edges(const uint8_t *px, int stride, int x, int y, const IntraArgs &a, const IntraState &s,
                            int *above, int *left, int *tmp, int rank, int n, Sync sync) {
  int w = 1 << a.log2W, h = 1 << a.log2H;
  for (int i = rank; i < w + h; i += n) {
    above[i] = above_sample(px, stride, x, y, a, i);
    left[i] = left_sample(px, stride, x, y, a, i);
  }
  if (rank == 0) above[-1] = left[-1] = corner_sample(px, stride, x, y, a);
  sync();
  if (!intra_is_directional(a.mode) || !a.edgeFilter) return;
  int pAngle = s.pAngle;
  if (pAngle != 90 && pAngle != 180) {
    if (pAngle > 90 && pAngle < 180 && (w + h) >= 24) {
      if (rank == 0) left[-1] = above[-1] = round2(left[0] * 5 + above[-1] * 6 + above[0] * 5, 4);
      sync();
    }
    for (int side = 0; side < 2; side++) {
      int *buf = side == 0 ? above : left;
      int have = side == 0 ? a.haveAbove : a.haveLeft;
      if (!have) continue;
      int strength = edge_strength(w, h, a.filterType, side == 0 ? pAngle - 90 : pAngle - 180);
      int sz = side == 0 ? imin(w, a.maxX - x + 1) + (pAngle < 90 ? h : 0) + 1
                         : imin(h, a.maxY - y + 1) + (pAngle > 180 ? w : 0) + 1;
      if (strength == 0) continue;
      for (int i = rank; i < sz; i += n) tmp[i] = buf[i - 1];
      sync();
      for (int i = 1 + rank; i < sz; i += n) {
        int acc = 0;
        for (int j = 0; j < 5; j++) acc += T(Intra_Edge_Kernel)[strength - 1][j] * tmp[clip3(0, sz - 1, i - 2 + j)];
        buf[i - 1] = (acc + 8) >> 4;
      }
      sync();
    }
  }
  for (int side = 0; side < 2; side++) {
    int up = side == 0 ? s.upAbove : s.upLeft;
    if (!up) continue;
    int *buf = side == 0 ? above : left;
    int numPx = side == 0 ? w + (pAngle < 90 ? h : 0) : h + (pAngle > 180 ? w : 0);
    if (rank == 0) {
      int dup[64 + 3];
      dup[0] = buf[-1];
      for (int i = -1; i < numPx; i++) dup[i + 2] = buf[i];
      dup[numPx + 2] = buf[numPx - 1];
      buf[-2] = dup[0];
      for (int i = 0; i < numPx; i++) {
        int v = -dup[i] + 9 * dup[i + 1] + 9 * dup[i + 2] - dup[i + 3];
        buf[2 * i - 1] = clip1(round2(v, 4));
        buf[2 * i] = dup[i + 2];
      }
    }
    sync();
  }
}

HD const int32_t *sm_weights(int log2) {
  if (log2 == 2) return T(Sm_Weights_Tx_4x4);
  if (log2 == 3) return T(Sm_Weights_Tx_8x8);
  if (log2 == 4) return T(Sm_Weights_Tx_16x16);
  if (log2 == 5) return T(Sm_Weights_Tx_32x32);
  return T(Sm_Weights_Tx_64x64);
}

// Intra prediction of sample (i, j) (row, column) from prepared edges.
HD int intra_pixel(const IntraArgs &a, const IntraState &s, const int *above, const int *left, int i, int j) {
  int w = 1 << a.log2W, h = 1 << a.log2H;
  int mode = a.mode;
  if (intra_is_directional(mode)) {
    int pAngle = s.pAngle, ua = s.upAbove, ul = s.upLeft;
    if (pAngle < 90) {
      int idx = (i + 1) * s.dx;
      int base = (idx >> (6 - ua)) + (j << ua);
      int shift = ((idx * (1 << ua)) >> 1) & 0x1F;
      int maxBaseX = (w + h - 1) << ua;
      if (base < maxBaseX) return round2(above[base] * (32 - shift) + above[base + 1] * shift, 5);
      return above[maxBaseX];
    } else if (pAngle > 90 && pAngle < 180) {
      int idx = (j << 6) - (i + 1) * s.dx;
      int base = idx >> (6 - ua);
      if (base >= -(1 << ua)) {
        int shift = ((idx * (1 << ua)) >> 1) & 0x1F;
        return round2(above[base] * (32 - shift) + above[base + 1] * shift, 5);
      }
      idx = (i << 6) - (j + 1) * s.dy;
      base = idx >> (6 - ul);
      int shift = ((idx * (1 << ul)) >> 1) & 0x1F;
      return round2(left[base] * (32 - shift) + left[base + 1] * shift, 5);
    } else if (pAngle > 180) {
      int idx = (j + 1) * s.dy;
      int base = (idx >> (6 - ul)) + (i << ul);
      int shift = ((idx * (1 << ul)) >> 1) & 0x1F;
      return round2(left[base] * (32 - shift) + left[base + 1] * shift, 5);
    } else if (pAngle == 90) {
      return above[j];
    }
    return left[i];
  }
  if (mode == SMOOTH_PRED) {
    const int32_t *wX = sm_weights(a.log2W), *wY = sm_weights(a.log2H);
    int v = wY[i] * above[j] + (256 - wY[i]) * left[h - 1] + wX[j] * left[i] + (256 - wX[j]) * above[w - 1];
    return round2(v, 9);
  }
  if (mode == SMOOTH_V_PRED) {
    const int32_t *wY = sm_weights(a.log2H);
    return round2(wY[i] * above[j] + (256 - wY[i]) * left[h - 1], 8);
  }
  if (mode == SMOOTH_H_PRED) {
    const int32_t *wX = sm_weights(a.log2W);
    return round2(wX[j] * left[i] + (256 - wX[j]) * above[w - 1], 8);
  }
  if (mode == PAETH_PRED) {
    int base = above[j] + left[i] - above[-1];
    int pLeft = iabs(base - left[i]), pTop = iabs(base - above[j]), pTopLeft = iabs(base - above[-1]);
    if (pLeft <= pTop && pLeft <= pTopLeft) return left[i];
    if (pTop <= pTopLeft) return above[j];
    return above[-1];
  }
  return -1;  // DC_PRED: computed once per block by intra_dc
}

// DC_PRED value of a block from its edges (spec 7.11.2.4 / 7.11.2.5).
HD int intra_dc(const IntraArgs &a, const int *above, const int *left) {
  int w = 1 << a.log2W, h = 1 << a.log2H;
  if (a.haveLeft && a.haveAbove) {
    int sum = 0;
    for (int k = 0; k < h; k++) sum += left[k];
    for (int k = 0; k < w; k++) sum += above[k];
    sum += (w + h) >> 1;
    return sum / (w + h);
  }
  if (a.haveLeft) {
    int sum = 0;
    for (int k = 0; k < h; k++) sum += left[k];
    return clip1((sum + (h >> 1)) >> a.log2H);
  }
  if (a.haveAbove) {
    int sum = 0;
    for (int k = 0; k < w; k++) sum += above[k];
    return clip1((sum + (w >> 1)) >> a.log2W);
  }
  return 1 << 7;
}

// ---- chroma from luma (spec 7.11.5) --------------------------------------------
// Scaled luma value of chroma sample (i, j): the 2x2 luma average x8 at the
// clamped luma position (MaxLumaW / MaxLumaH rule).
HD int cfl_luma(const uint8_t *luma, int lumaStride, int startX, int startY, int maxLumaW, int maxLumaH, int i,
                int j) {
  int ly = imin((startY + i) << 1, maxLumaH - 2);
  int lx = imin((startX + j) << 1, maxLumaW - 2);
  const uint8_t *l = luma + ly * lumaStride + lx;
  return ((int)l[0] + l[1] + l[lumaStride] + l[lumaStride + 1]) << 1;
}

HD int cfl_pixel(int dc, int alpha, int v, int avg) { return clip3(0, 255, dc + round2signed(alpha * (v - avg), 6)); }

}  // namespace pred
