// In-loop filters: loop-filter info, deblocking (spec 7.14), CDEF
// (spec 7.15) with per-superblock preset selection, loop restoration apply
// (spec 7.17). Reference: src/kernels/k_lf.h, k_cdef.h, k_lr.h, the filter
// stage of src/backend_cpu.c:158-188 and the host helpers build_filter_info
// and cdef_select (src/encoder.c:513-563).
//
// B200 mapping. Deblocking: one thread per (plane, edge, sample line); the
// spec makes the edges of one pass independent (a filter never reaches the
// samples another edge of the same pass modifies), so a pass is one launch.
// CDEF: one 64-thread CTA per 8x8 block: the direction search accumulates
// its partial sums in shared memory, then each thread filters one luma
// sample (and one chroma sample) for every preset. Preset selection: one CTA
// per superblock reduces the SSE of every preset and copies the winner into
// the reconstruction. Loop restoration: one thread per 4x4 block.
#pragma once

#include "common.cuh"

namespace flt {

// ---- loop filter info (encoder.c:513-526) --------------------------------------------
__global__ void k_filter_info(const FrameParams *fp, const BlockInfo *blocks, const SbInfo *sbs, uint8_t *info) {
  int sb = blockIdx.x, k = threadIdx.x;
  if (k >= sbs[sb].num_blocks) return;
  const BlockInfo *b = &blocks[sbs[sb].first_block + k];
  int skip = b->eob[0] == 0 && b->eob[1] == 0 && b->eob[2] == 0;
  int bw4 = T(Num_4x4_Blocks_Wide)[b->bsize], bh4 = T(Num_4x4_Blocks_High)[b->bsize];
  uint8_t v = (uint8_t)(b->bsize | (skip << 5) | (b->tx_depth << 6));
  for (int y = 0; y < bh4 && b->mi_row + y < fp->mi_rows; y++)
    for (int x = 0; x < bw4 && b->mi_col + x < fp->mi_cols; x++) info[(b->mi_row + y) * fp->mi_cols + b->mi_col + x] = v;
}

// ---- deblocking (k_lf.h:13-136) ---------------------------------------------------
HD int lf_tx_size(int info, int plane) {
  return plane == 0 ? depth_tx_size(info & 31, (info >> 6) & 3) : uv_tx_size(info & 31, 1, 1);
}

__device__ void lf_sample(uint8_t *px, int pitch, int plane, int lvl, int sharp, int filterSize) {
  int shift = sharp > 4 ? 2 : (sharp > 0 ? 1 : 0);
  int limit = sharp > 0 ? clip3(1, 9 - sharp, lvl >> shift) : imax(1, lvl >> shift);
  int blimit = 2 * (lvl + 2) + limit;
  int thresh = lvl >> 4;
#define S(k) ((int)px[(k) * pitch])
  int q0 = S(0), q1 = S(1), p0 = S(-1), p1 = S(-2);
  int filterLen = filterSize == 4 ? 4 : (plane != 0 ? 6 : (filterSize == 8 ? 8 : 16));
  int q2 = 0, q3 = 0, p2 = 0, p3 = 0;
  if (filterLen >= 6 || filterSize >= 8) {
    q2 = S(2);
    p2 = S(-3);
  }
  if (filterLen >= 8) {
    q3 = S(3);
    p3 = S(-4);
  }
  int hevMask = (iabs(p1 - p0) > thresh) || (iabs(q1 - q0) > thresh);
  int mask = 0;
  mask |= iabs(p1 - p0) > limit;
  mask |= iabs(q1 - q0) > limit;
  mask |= iabs(p0 - q0) * 2 + iabs(p1 - q1) / 2 > blimit;
  if (filterLen >= 6) {
    mask |= iabs(p2 - p1) > limit;
    mask |= iabs(q2 - q1) > limit;
  }
  if (filterLen >= 8) {
    mask |= iabs(p3 - p2) > limit;
    mask |= iabs(q3 - q2) > limit;
  }
  if (mask) return;
  int flatMask = 0, flatMask2 = 0;
  if (filterSize >= 8) {
    int m = 0;
    m |= iabs(p1 - p0) > 1;
    m |= iabs(q1 - q0) > 1;
    m |= iabs(p2 - p0) > 1;
    m |= iabs(q2 - q0) > 1;
    if (filterLen >= 8) {
      m |= iabs(p3 - p0) > 1;
      m |= iabs(q3 - q0) > 1;
    }
    flatMask = m == 0;
  }
  if (filterSize >= 16) {
    int q4 = S(4), q5 = S(5), q6 = S(6), p4 = S(-5), p5 = S(-6), p6 = S(-7);
    int m = 0;
    m |= iabs(p6 - p0) > 1;
    m |= iabs(q6 - q0) > 1;
    m |= iabs(p5 - p0) > 1;
    m |= iabs(q5 - q0) > 1;
    m |= iabs(p4 - p0) > 1;
    m |= iabs(q4 - q0) > 1;
    flatMask2 = m == 0;
  }
  if (filterSize == 4 || !flatMask) {
    int ps1 = p1 - 128, ps0 = p0 - 128, qs0 = q0 - 128, qs1 = q1 - 128;
    int filter = hevMask ? clip3(-128, 127, ps1 - qs1) : 0;
    filter = clip3(-128, 127, filter + 3 * (qs0 - ps0));
    int filter1 = clip3(-128, 127, filter + 4) >> 3;
    int filter2 = clip3(-128, 127, filter + 3) >> 3;
    px[0] = (uint8_t)(clip3(-128, 127, qs0 - filter1) + 128);
    px[-pitch] = (uint8_t)(clip3(-128, 127, ps0 + filter2) + 128);
    if (!hevMask) {
      filter = round2(filter1, 1);
      px[pitch] = (uint8_t)(clip3(-128, 127, qs1 - filter) + 128);
      px[-2 * pitch] = (uint8_t)(clip3(-128, 127, ps1 + filter) + 128);
    }
  } else {
    int log2Size = (filterSize == 8 || !flatMask2) ? 3 : 4;
    int n = log2Size == 4 ? 6 : (plane == 0 ? 3 : 2);
    int n2 = (log2Size == 3 && plane == 0) ? 0 : 1;
    int v[14];
    for (int k = -(n + 1); k <= n; k++) v[k + 7] = S(k);
    int F[12];
    for (int i = -n; i < n; i++) {
      int t = 0;
      for (int j = -n; j <= n; j++) {
        int p = clip3(-(n + 1), n, i + j);
        int tap = iabs(j) <= n2 ? 2 : 1;
        t += v[p + 7] * tap;
      }
      F[i + n] = round2(t, log2Size);
    }
    for (int i = -n; i < n; i++) px[i * pitch] = (uint8_t)F[i + n];
  }
#undef S
}

// One pass (0: vertical edges, 1: horizontal edges); thread per (plane,
// line, edge position k, sample i).
__global__ void k_deblock(const FrameParams *fp, uint8_t *rec, const uint8_t *miSizes, int pass) {
  int lines = pass == 0 ? fp->mi_rows : fp->mi_cols;
  int n = pass == 0 ? fp->mi_cols : fp->mi_rows;
  long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  long long per = (long long)lines * n * 4;
  if (g >= 3 * per) return;
  int plane = (int)(g / per);
  long long rem = g % per;
  int line = (int)(rem / (n * 4)), k = (int)((rem / 4) % n), i = (int)(rem & 3);
  int sub = plane > 0;
  if (sub && ((line & 1) || (k & 1))) return;
  int lvl = clip3(0, MAX_LOOP_FILTER, fp->lf_level[plane == 0 ? pass : plane + 1]);
  if (lvl == 0) return;
  int stride = fp->stride[plane];
  uint8_t *base = rec + fp->offset[plane];
  int dx = pass == 0, dy = pass == 1;
  int row0 = pass == 0 ? line : k, col0 = pass == 0 ? k : line;
  int x = col0 * MI_SIZE, y = row0 * MI_SIZE;
  int row = row0 | sub, col = col0 | sub;
  if (x >= fp->frame_w || y >= fp->frame_h) return;
  if (pass == 0 && x == 0) return;
  if (pass == 1 && y == 0) return;
  int xP = x >> sub, yP = y >> sub;
  int prevRow = row - (dy << sub), prevCol = col - (dx << sub);
  int txSz = lf_tx_size(miSizes[row * fp->mi_cols + col], plane);
  int prevTxSz = lf_tx_size(miSizes[prevRow * fp->mi_cols + prevCol], plane);
  int isTxEdge = pass == 0 ? (xP % T(Tx_Width)[txSz]) == 0 : (yP % T(Tx_Height)[txSz]) == 0;
  if (!isTxEdge) return;
  int baseSize = pass == 0 ? imin(T(Tx_Width)[prevTxSz], T(Tx_Width)[txSz]) : imin(T(Tx_Height)[prevTxSz], T(Tx_Height)[txSz]);
  int filterSize = plane == 0 ? imin(16, baseSize) : imin(8, baseSize);
  int sx = xP + dy * i, sy = yP + dx * i;
  WORK(W_LF_TAPS, filterSize == 4 ? 4 : (plane != 0 ? 6 : (filterSize == 8 ? 8 : 16)));  // the line's filter length
  lf_sample(base + sy * stride + sx, pass == 0 ? 1 : stride, plane, lvl, fp->lf_sharpness, filterSize);
}

// ---- CDEF (k_cdef.h:9-150) ------------------------------------------------------------
__device__ __forceinline__ int cdef_constrain(int diff, int threshold, int damping) {
  if (!threshold) return 0;
  int dampingAdj = imax(0, damping - floor_log2(threshold));
  int sign = diff < 0 ? -1 : 1;
  return sign * clip3(0, iabs(diff), threshold - (iabs(diff) >> dampingAdj));
}

// Filtered value of sample (i, j) of the 8x8 (4x4 chroma) block at mi (r, c).
__device__ int cdef_pixel(const FrameParams *fp, const uint8_t *cur, int plane, int r, int c, int i, int j, int priStr,
                          int secStr, int damping, int dir) {
  int sub = plane > 0, stride = fp->stride[plane];
  const uint8_t *src = cur + fp->offset[plane];
  int x0 = (c * MI_SIZE) >> sub, y0 = (r * MI_SIZE) >> sub;
  int sum = 0;
  int x = src[(y0 + i) * stride + x0 + j];
  int mx = x, mn = x;
  for (int k = 0; k < 2; k++)
    for (int sign = -1; sign <= 1; sign += 2)
      for (int t = 0; t < 3; t++) {
        int d = t == 0 ? dir : ((dir + (t == 1 ? -2 : 2)) & 7);
        int yy = y0 + i + sign * T(Cdef_Directions)[d][k][0];
        int xx = x0 + j + sign * T(Cdef_Directions)[d][k][1];
        int candR = (yy * (1 << sub)) >> 2, candC = (xx * (1 << sub)) >> 2;
        if (!(candC >= 0 && candC < fp->mi_cols && candR >= 0 && candR < fp->mi_rows)) continue;
        int p = src[yy * stride + xx];
        if (t == 0) sum += T(Cdef_Pri_Taps)[priStr & 1][k] * cdef_constrain(p - x, priStr, damping);
        else sum += T(Cdef_Sec_Taps)[priStr & 1][k] * cdef_constrain(p - x, secStr, damping);
        mx = imax(p, mx);
        mn = imin(p, mn);
      }
  return clip3(mn, mx, x + ((8 + sum - (sum < 0)) >> 4));
}

// One CTA of 64 threads per 8x8 block (mi rows / cols in steps of 2): the
// direction once, then every preset's output into out + k * frameBytes.
__global__ void __launch_bounds__(64) k_cdef(const FrameParams *fp, const uint8_t *cur, uint8_t *out,
                                             long long frameBytes, const uint8_t *info, int npresets) {
  __shared__ int partial[8][15];
  __shared__ int cost[8];
  __shared__ int s_dir, s_var;
  int bc = (fp->mi_cols + 1) >> 1;
  int r = (blockIdx.x / bc) * 2, c = (blockIdx.x % bc) * 2;
  int tid = threadIdx.x;
  int skip = (info[r * fp->mi_cols + c] >> 5) & 1;
  if (tid == 0 && !skip) WORK(W_CDEF_TAPS, 64 * 8);  // direction search: 64 samples into 8 projections
  if (!skip) {
    for (int k = tid; k < 8 * 15; k += 64) partial[k / 15][k % 15] = 0;
    __syncthreads();
    int i = tid >> 3, j = tid & 7;
    int x = (int)cur[fp->offset[0] + (r * MI_SIZE + i) * fp->stride[0] + c * MI_SIZE + j] - 128;
    atomicAdd(&partial[0][i + j], x);
    atomicAdd(&partial[1][i + j / 2], x);
    atomicAdd(&partial[2][i], x);
    atomicAdd(&partial[3][3 + i - j / 2], x);
    atomicAdd(&partial[4][7 + i - j], x);
    atomicAdd(&partial[5][3 - i / 2 + j], x);
    atomicAdd(&partial[6][j], x);
    atomicAdd(&partial[7][i / 2 + j], x);
    __syncthreads();
    if (tid < 8) {
      int d = tid, cst = 0;
      if (d == 2 || d == 6) {
        for (int k = 0; k < 8; k++) cst += partial[d][k] * partial[d][k];
        cst *= T(Div_Table)[8];
      } else if (d == 0 || d == 4) {
        for (int k = 0; k < 7; k++)
          cst += (partial[d][k] * partial[d][k] + partial[d][14 - k] * partial[d][14 - k]) * T(Div_Table)[k + 1];
        cst += partial[d][7] * partial[d][7] * T(Div_Table)[8];
      } else {
        for (int k = 0; k < 5; k++) cst += partial[d][3 + k] * partial[d][3 + k];
        cst *= T(Div_Table)[8];
        for (int k = 0; k < 3; k++)
          cst += (partial[d][k] * partial[d][k] + partial[d][10 - k] * partial[d][10 - k]) * T(Div_Table)[2 * k + 2];
      }
      cost[d] = cst;
    }
    __syncthreads();
    if (tid == 0) {
      int best = 0, dir = 0;
      for (int d = 0; d < 8; d++)
        if (cost[d] > best) {
          best = cost[d];
          dir = d;
        }
      s_dir = dir;
      s_var = (best - cost[(dir + 4) & 7]) >> 10;
    }
    __syncthreads();
  }
  int yDir = skip ? 0 : s_dir, var = skip ? 0 : s_var;
  for (int idx = 0; idx < npresets; idx++) {
    uint8_t *o = out + (long long)idx * frameBytes;
    int priStr = fp->cdef_y_pri[idx], secStr = fp->cdef_y_sec[idx];
    int uvPri = fp->cdef_uv_pri[idx], uvSec = fp->cdef_uv_sec[idx];
    int copyOnly = skip || (priStr == 0 && secStr == 0 && uvPri == 0 && uvSec == 0);
    if (tid == 0 && !copyOnly) WORK(W_CDEF_TAPS, (64 + 32) * 12);  // 12 taps per filtered sample
    // luma sample tid; chroma samples tid < 32 (16 per plane)
    {
      int i = tid >> 3, j = tid & 7, stride = fp->stride[0];
      size_t off = fp->offset[0] + (size_t)(r * MI_SIZE + i) * stride + c * MI_SIZE + j;
      int v;
      if (copyOnly) {
        v = cur[off];
      } else {
        int dir = priStr == 0 ? 0 : yDir;
        int varStr = (var >> 6) ? imin(floor_log2(var >> 6), 12) : 0;
        int pri = var ? (priStr * (4 + varStr) + 8) >> 4 : 0;
        v = cdef_pixel(fp, cur, 0, r, c, i, j, pri, secStr, fp->cdef_damping, dir);
      }
      o[off] = (uint8_t)v;
    }
    if (tid < 32) {
      int plane = 1 + (tid >> 4), i = (tid >> 2) & 3, j = tid & 3, stride = fp->stride[plane];
      size_t off = fp->offset[plane] + (size_t)((r * MI_SIZE >> 1) + i) * stride + (c * MI_SIZE >> 1) + j;
      int v;
      if (copyOnly) {
        v = cur[off];
      } else {
        int dir = uvPri == 0 ? 0 : T(Cdef_Uv_Dir)[1][1][yDir];
        v = cdef_pixel(fp, cur, plane, r, c, i, j, uvPri, uvSec, fp->cdef_damping - 1, dir);
      }
      o[off] = (uint8_t)v;
    }
  }
}

// Per superblock: SSE of every preset against the source (real frame area),
// first minimum, copy of the winner into rec (mi-aligned area)
// (cdef_select, encoder.c:530-563).
__global__ void __launch_bounds__(256) k_cdef_select(const FrameParams *fp, const uint8_t *src, const uint8_t *cdefbuf,
                                                     long long frameBytes, uint8_t *rec, int8_t *choice, int npresets) {
  __shared__ long long red[8][4];
  __shared__ int s_best;
  int sb = blockIdx.x;
  int sr = sb / fp->sb_cols, sc = sb % fp->sb_cols;
  int tid = threadIdx.x;
  long long sse[4] = {0, 0, 0, 0};
  for (int p = 0; p < 3; p++) {
    int sub = p > 0, n = 64 >> sub;
    int pw = p ? (fp->frame_w + 1) >> 1 : fp->frame_w, ph = p ? (fp->frame_h + 1) >> 1 : fp->frame_h;
    for (int k = tid; k < n * n; k += 256) {
      int y = sr * n + k / n, x = sc * n + k % n;
      if (y >= ph || x >= pw) continue;
      size_t o = fp->offset[p] + (size_t)y * fp->stride[p] + x;
      int s = src[o];
      for (int q = 0; q < npresets; q++) {
        int d = (int)cdefbuf[(size_t)q * frameBytes + o] - s;
        sse[q] += d * d;
      }
    }
  }
  for (int q = 0; q < npresets; q++) {
    long long v = sse[q];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if ((tid & 31) == 0) red[tid >> 5][q] = v;
  }
  __syncthreads();
  if (tid == 0) {
    long long best = -1;
    int bestK = 0;
    for (int q = 0; q < npresets; q++) {
      long long s = 0;
      for (int w = 0; w < 8; w++) s += red[w][q];
      if (best < 0 || s < best) {
        best = s;
        bestK = q;
      }
    }
    s_best = bestK;
    choice[sb] = (int8_t)bestK;
  }
  __syncthreads();
  const uint8_t *out = cdefbuf + (size_t)s_best * frameBytes;
  for (int p = 0; p < 3; p++) {
    int sub = p > 0, n = 64 >> sub;
    int mw = (fp->mi_cols * 4) >> sub, mh = (fp->mi_rows * 4) >> sub;
    for (int k = tid; k < n * n; k += 256) {
      int y = sr * n + k / n, x = sc * n + k % n;
      if (y >= mh || x >= mw) continue;
      size_t o = fp->offset[p] + (size_t)y * fp->stride[p] + x;
      rec[o] = out[o];
    }
  }
}

// ---- loop restoration apply (k_lr.h:28-202) ----------------------------------------------
struct LrBlock {
  int x, y, w, h;
  int stripeStart, stripeEnd;
  int planeEndX, planeEndY;
  int unitRow, unitCol;
};

HD int lr_block_setup(const FrameParams *fp, int plane, int row, int col, LrBlock *lb) {
  int sub = plane > 0;
  int lumaY = row * MI_SIZE;
  int stripeNum = (lumaY + 8) / 64;
  lb->stripeStart = (-8 + stripeNum * 64) >> sub;
  lb->stripeEnd = lb->stripeStart + (64 >> sub) - 1;
  int unitSize = fp->lr_unit_size[plane];
  lb->unitRow = imin(fp->lr_unit_rows[plane] - 1, ((row * MI_SIZE + 8) >> sub) / unitSize);
  lb->unitCol = imin(fp->lr_unit_cols[plane] - 1, ((col * MI_SIZE) >> sub) / unitSize);
  lb->planeEndX = ((fp->frame_w + sub) >> sub) - 1;
  lb->planeEndY = ((fp->frame_h + sub) >> sub) - 1;
  lb->x = (col * MI_SIZE) >> sub;
  lb->y = (row * MI_SIZE) >> sub;
  lb->w = imin(MI_SIZE >> sub, lb->planeEndX - lb->x + 1);
  lb->h = imin(MI_SIZE >> sub, lb->planeEndY - lb->y + 1);
  return lb->w > 0 && lb->h > 0;
}

// get_source_sample( ) (spec 7.17.6)
HD int lr_src(const FrameParams *fp, int plane, const LrBlock *lb, const uint8_t *cdef, const uint8_t *dbk, int x, int y) {
  x = imax(0, imin(lb->planeEndX, x));
  y = imax(0, imin(lb->planeEndY, y));
  int stride = fp->stride[plane];
  if (y < lb->stripeStart) {
    y = imax(lb->stripeStart - 2, y);
    return dbk[fp->offset[plane] + y * stride + x];
  } else if (y > lb->stripeEnd) {
    y = imin(lb->stripeEnd + 2, y);
    return dbk[fp->offset[plane] + y * stride + x];
  }
  return cdef[fp->offset[plane] + y * stride + x];
}

// The samples the loop-restoration filters read: get_source_sample( ) for
// the filter taps, and the CDEF output at the block's own positions. FrameSrc
// reads the frame buffers; the parameter search reads shared-memory windows
// (lrs::WinSrc) through the same filter code.
struct FrameSrc {
  const FrameParams *fp;
  int plane;
  const uint8_t *cdef, *dbk;
  HD int tap(const LrBlock *lb, int x, int y) const { return lr_src(fp, plane, lb, cdef, dbk, x, y); }
  HD int own(int x, int y) const { return cdef[fp->offset[plane] + y * fp->stride[plane] + x]; }
};

// Output of the filters: sink(x, y, value) for plane sample (x, y). The apply
// kernel stores it, the parameter search accumulates its squared error.
struct StoreSink {
  const FrameParams *fp;
  int plane;
  uint8_t *out;
  HD void operator()(int x, int y, int v) { out[fp->offset[plane] + y * fp->stride[plane] + x] = (uint8_t)v; }
};

// Wiener filter (spec 7.17.4, 8-bit rounding).
template <class Src, class Sink>
HD void lr_wiener_to(const LrBlock *lb, const Src &in, const LrUnit *u, Sink &sink) {
  int vf[7], hf[7];
  vf[3] = 128;
  hf[3] = 128;
  for (int i = 0; i < 3; i++) {
    vf[i] = vf[6 - i] = u->wiener[0][i];
    vf[3] -= 2 * u->wiener[0][i];
    hf[i] = hf[6 - i] = u->wiener[1][i];
    hf[3] -= 2 * u->wiener[1][i];
  }
  const int round0 = 3, round1 = 11;
  int offset = 1 << (8 + FILTER_BITS - round0 - 1);
  int limit = (1 << (8 + 1 + FILTER_BITS - round0)) - 1;
  int inter[10][4];
  for (int r = 0; r < lb->h + 6; r++)
    for (int c = 0; c < lb->w; c++) {
      int s = 0;
      for (int t = 0; t < 7; t++) s += hf[t] * in.tap(lb, lb->x + c + t - 3, lb->y + r - 3);
      inter[r][c] = clip3(-offset, limit - offset, round2(s, round0));
    }
  for (int r = 0; r < lb->h; r++)
    for (int c = 0; c < lb->w; c++) {
      int s = 0;
      for (int t = 0; t < 7; t++) s += vf[t] * inter[r + t][c];
      sink(lb->x + c, lb->y + r, clip3(0, 255, round2(s, round1)));
    }
}

HD void lr_wiener(const FrameParams *fp, int plane, const LrBlock *lb, const uint8_t *cdef, const uint8_t *dbk,
                  uint8_t *out, const LrUnit *u) {
  FrameSrc in{fp, plane, cdef, dbk};
  StoreSink sink{fp, plane, out};
  lr_wiener_to(lb, in, u, sink);
}

// Box filter (spec 7.17.3); F gets w x h values (row stride 4).
template <class Src>
HD void lr_box(const LrBlock *lb, const Src &in, int set, int pass, int *F) {
  int r = T(Sgr_Params)[set][pass * 2 + 0];
  if (r == 0) return;
  int eps = T(Sgr_Params)[set][pass * 2 + 1];
  int A[6][6], Bv[6][6];
  int n = (2 * r + 1) * (2 * r + 1);
  int n2e = n * n * eps;
  int s = ((1 << SGRPROJ_MTABLE_BITS) + n2e / 2) / n2e;
  int oneOverN = ((1 << SGRPROJ_RECIP_BITS) + (n / 2)) / n;
  for (int i = -1; i < lb->h + 1; i++)
    for (int j = -1; j < lb->w + 1; j++) {
      long long a = 0, b = 0;
      for (int dy = -r; dy <= r; dy++)
        for (int dx = -r; dx <= r; dx++) {
          long long c = in.tap(lb, lb->x + j + dx, lb->y + i + dy);
          a += c * c;
          b += c;
        }
      long long d = b;
      long long p = a * n - d * d;
      if (p < 0) p = 0;
      long long z = (p * s + (1LL << (SGRPROJ_MTABLE_BITS - 1))) >> SGRPROJ_MTABLE_BITS;
      long long a2;
      if (z >= 255) a2 = 256;
      else if (z == 0) a2 = 1;
      else a2 = ((z << SGRPROJ_SGR_BITS) + (z / 2)) / (z + 1);
      long long b2 = ((1LL << SGRPROJ_SGR_BITS) - a2) * b * oneOverN;
      A[i + 1][j + 1] = (int)a2;
      Bv[i + 1][j + 1] = (int)((b2 + (1LL << (SGRPROJ_RECIP_BITS - 1))) >> SGRPROJ_RECIP_BITS);
    }
  for (int i = 0; i < lb->h; i++) {
    int shift = 5;
    if (pass == 0 && (i & 1)) shift = 4;
    for (int j = 0; j < lb->w; j++) {
      long long a = 0, b = 0;
      for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
          int weight;
          if (pass == 0) weight = ((i + dy) & 1) ? (dx == 0 ? 6 : 5) : 0;
          else weight = (dx == 0 || dy == 0) ? 4 : 3;
          a += weight * A[i + dy + 1][j + dx + 1];
          b += weight * Bv[i + dy + 1][j + dx + 1];
        }
      long long v = a * in.own(lb->x + j, lb->y + i) + b;
      int sh = SGRPROJ_SGR_BITS + shift - SGRPROJ_RST_BITS;
      F[i * 4 + j] = (int)((v + (1LL << (sh - 1))) >> sh);
    }
  }
}

// Self-guided projection (spec 7.17.2) of a block whose box-filter outputs
// are flt0 / flt1.
template <class Src, class Sink>
HD void lr_sgr_project(const LrBlock *lb, const Src &in, const LrUnit *u, const int *flt0, const int *flt1, Sink &sink) {
  int w0 = u->xqd[0], w1 = u->xqd[1];
  int w2 = (1 << SGRPROJ_PRJ_BITS) - w0 - w1;
  int r0 = T(Sgr_Params)[u->set][0], r1 = T(Sgr_Params)[u->set][2];
  for (int i = 0; i < lb->h; i++)
    for (int j = 0; j < lb->w; j++) {
      int uu = in.own(lb->x + j, lb->y + i) << SGRPROJ_RST_BITS;
      int v = w1 * uu;
      v += r0 ? w0 * flt0[i * 4 + j] : w0 * uu;
      v += r1 ? w2 * flt1[i * 4 + j] : w2 * uu;
      sink(lb->x + j, lb->y + i, clip3(0, 255, round2(v, SGRPROJ_RST_BITS + SGRPROJ_PRJ_BITS)));
    }
}

// Self-guided filter (spec 7.17.2).
HD void lr_sgr(const FrameParams *fp, int plane, const LrBlock *lb, const uint8_t *cdef, const uint8_t *dbk, uint8_t *out,
               const LrUnit *u) {
  FrameSrc in{fp, plane, cdef, dbk};
  int flt0[16], flt1[16];
  lr_box(lb, in, u->set, 0, flt0);
  lr_box(lb, in, u->set, 1, flt1);
  StoreSink sink{fp, plane, out};
  lr_sgr_project(lb, in, u, flt0, flt1, sink);
}

// Thread per (plane, 4x4 luma block): loop_restore_block( ) with the unit's
// filter, RESTORE_NONE copies the CDEF output.
__global__ void k_lr_apply(const FrameParams *fp, const uint8_t *cdef, const uint8_t *dbk, uint8_t *out,
                           const LrUnit *units) {
  int rows4 = (fp->frame_h + 3) >> 2, cols4 = (fp->frame_w + 3) >> 2, n = rows4 * cols4;
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= 3 * n) return;
  int plane = g / n, i = g % n;
  LrBlock lb;
  if (!lr_block_setup(fp, plane, i / cols4, i % cols4, &lb)) return;
  LrUnit u;
  if (fp->lr_type[plane] == RESTORE_NONE) u.type = RESTORE_NONE;
  else u = units[fp->lr_unit_off[plane] + lb.unitRow * fp->lr_unit_cols[plane] + lb.unitCol];
  WORK(W_LR_TAPS, lb.w * lb.h * (u.type == RESTORE_WIENER ? 14 : u.type == RESTORE_SGRPROJ ? 34 : 0));
  if (u.type == RESTORE_WIENER) {
    lr_wiener(fp, plane, &lb, cdef, dbk, out, &u);
  } else if (u.type == RESTORE_SGRPROJ) {
    lr_sgr(fp, plane, &lb, cdef, dbk, out, &u);
  } else {
    int stride = fp->stride[plane];
    for (int y = 0; y < lb.h; y++)
      for (int x = 0; x < lb.w; x++) {
        int o = fp->offset[plane] + (lb.y + y) * stride + lb.x + x;
        out[o] = cdef[o];
      }
  }
}

}  // namespace flt
