// Hierarchical motion search (reference src/kernels/k_me.h, driven by
// src/backend_cpu.c:23-56).
//
// Per node (64x64 .. 8x8 square of a superblock) and reference: an ordered
// list of full-pel candidates (level 0: a coarse grid, optionally on the
// 4x4-decimated planes, then refinement stages), the first minimum of
// SAD + ac_q * bits / 64, then half- and quarter-pel refinement by the first
// minimum of the 4x4-SATD over the node. The levels depend on each other
// (children search around the parent's vector) and run as separate launches.
//
// B200 mapping: one warp per (node, reference). Lanes take candidates (SAD
// rows on packed bytes with __vsadu4; interior candidates read unaligned
// words through funnel shifts), and the warp reduces the 64-bit key
// (cost << 32 | index) with shuffles, which yields exactly the serial first
// minimum. The 64x64 level has few nodes: a CTA per node, its four warps
// taking candidates in turn and each warp's lanes splitting a candidate's
// byte pairs. Sub-pel candidates x 4x4 units are spread over the lanes and
// summed in shared memory. Quarter-pel planes (16 per reference, EIGHTTAP,
// the T_ME_HPEL mode) are built once per reference picture by their own
// kernel, one thread per sample.
#pragma once

#include "common.cuh"
#include "pred.cuh"

namespace me {

struct Frame {
  const FrameParams *fp;   // device copy
  const uint8_t *src;      // padded source frame
  const uint8_t *ref;      // reference frame (padded layout)
  const uint8_t *qp;       // 16 quarter-pel planes of ref, frame_w x frame_h each
  const uint8_t *dsrc;     // decimated source, dec_w x dec_h
  const uint8_t *dref;     // decimated reference
  int32_t *mv;             // mv field of this reference
  int isGold;
};

HD int dec_w(const FrameParams *fp) { return (fp->frame_w + 3) >> 2; }
HD int dec_h(const FrameParams *fp) { return (fp->frame_h + 3) >> 2; }

// ---- quarter-pel and decimated planes -----------------------------------------

// Plane fy * 4 + fx holds the EIGHTTAP prediction of (y + fy / 4, x + fx / 4)
// (k_me.h:289-313): horizontal Round2( ., 3 ), vertical Round2( ., 11 ), Clip1.
// A CTA of 32 x 8 threads makes a QP_TW x QP_TH tile of all 16 planes: the
// clamped reference window (QP_TH + 7 rows, QP_TW + 7 columns) is staged in
// shared memory once, the horizontal pass (4 phases) runs once per window
// row and column, and each thread forms 4 consecutive samples of one row for
// every plane, stored as one 32-bit word where the plane row allows. Every
// sample is the same sums and roundings as the per-sample definition.
constexpr int QP_TW = 128, QP_TH = 8, QP_THREADS = 256;

__global__ void __launch_bounds__(QP_THREADS) k_qpel_planes(const FrameParams *fp, const uint8_t *ref, uint8_t *qp) {
  __shared__ uint8_t win[QP_TH + 7][QP_TW + 8];
  __shared__ __align__(16) int16_t hs[4][QP_TH + 7][QP_TW];
  const int W = fp->frame_w, H = fp->frame_h, stride = fp->stride[0];
  const uint8_t *rp = ref + fp->offset[0];
  const int x0 = blockIdx.x * QP_TW, y0 = blockIdx.y * QP_TH, tid = threadIdx.x;
  for (int i = tid; i < (QP_TH + 7) * (QP_TW + 7); i += QP_THREADS) {
    int r = i / (QP_TW + 7), c = i - r * (QP_TW + 7);
    win[r][c] = rp[clip3(0, H - 1, y0 + r - 3) * stride + clip3(0, W - 1, x0 + c - 3)];
  }
  __syncthreads();
  for (int i = tid; i < (QP_TH + 7) * QP_TW; i += QP_THREADS) {
    int r = i / QP_TW, x = i - r * QP_TW;
    int px[8];
    for (int u = 0; u < 8; u++) px[u] = win[r][x + u];
    for (int fx = 0; fx < 4; fx++) {
      const int32_t *f = d_Subpel_Filters[EIGHTTAP][4 * fx];
      int sum = 0;
      for (int u = 0; u < 8; u++) sum += f[u] * px[u];
      hs[fx][r][x] = (int16_t)round2(sum, 3);
    }
  }
  __syncthreads();
  // taps: the horizontal pass over the window (4 phases), the vertical pass per output of 16 planes
  if (tid == 0) WORK(W_QPEL_TAPS, (QP_TH + 7) * QP_TW * 4 * 8 + imin(QP_TH, H - y0) * imin(QP_TW, W - x0) * 16 * 8);
  const int ty = tid >> 5, xx = (tid & 31) * 4, y = y0 + ty, x = x0 + xx;
  if (y >= H || x >= W) return;
  const size_t n = (size_t)W * H, o = (size_t)y * W + x;
  const bool word = (W & 3) == 0 && x + 3 < W;  // 4-byte aligned and inside the row
  for (int fx = 0; fx < 4; fx++) {
    // this thread's 8 rows x 4 columns of horizontal sums, one 8-byte load per row
    int hv[8][4];
    for (int t = 0; t < 8; t++) {
      int2 w2 = *(const int2 *)&hs[fx][ty + t][xx];
      hv[t][0] = (int16_t)(w2.x & 0xffff);
      hv[t][1] = (int16_t)(w2.x >> 16);
      hv[t][2] = (int16_t)(w2.y & 0xffff);
      hv[t][3] = (int16_t)(w2.y >> 16);
    }
    for (int fy = 0; fy < 4; fy++) {
      const int32_t *f = d_Subpel_Filters[EIGHTTAP][4 * fy];
      uint8_t *plane = qp + (size_t)(fy * 4 + fx) * n;
      uint32_t packed = 0;
      for (int k = 0; k < 4; k++) {
        int sum = 0;
        for (int t = 0; t < 8; t++) sum += f[t] * hv[t][k];
        uint32_t v = (uint32_t)clip1(round2(sum, 11));
        if (word) packed |= v << (8 * k);
        else if (x + k < W) plane[o + k] = (uint8_t)v;
      }
      if (word) *(uint32_t *)(plane + o) = packed;
    }
  }
}

// 4x4 average of the frame, (sum + 8) >> 4 (k_me.h:112-118).
__global__ void k_dec_plane(const FrameParams *fp, const uint8_t *pl, uint8_t *out) {
  int W = dec_w(fp), H = dec_h(fp);
  int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= W || y >= H) return;
  int s = 0;
  for (int i = 0; i < 4; i++)
    for (int j = 0; j < 4; j++)
      s += pl[fp->offset[0] + clip3(0, fp->frame_h - 1, 4 * y + i) * fp->stride[0] + clip3(0, fp->frame_w - 1, 4 * x + j)];
  out[(size_t)y * W + x] = (uint8_t)((s + 8) >> 4);
}

// ---- search node ----------------------------------------------------------------
struct Node {
  int valid, x, y, w;
  int cy, cx, range, step, stages, count;
  int pr, pc, copy;
};

#define ME_COARSE_STEP 4
#define ME_REFINE 3

__device__ __forceinline__ int leaf_no8(const FrameParams *fp) {
  return (fp->turbo & T_LEAF_NO8) && fp->leaf && !fp->frame_is_intra;
}

// Node setup (k_me.h:141-178).
__device__ Node make_node(const FrameParams *fp, int sb, int level, int i, const int32_t *mv) {
  Node m;
  int sbRow = sb / fp->sb_cols, sbCol = sb % fp->sb_cols, n = 1 << level;
  m.w = 64 >> level;
  m.x = sbCol * 64 + (i % n) * m.w;
  m.y = sbRow * 64 + (i / n) * m.w;
  m.valid = m.x < fp->frame_w && m.y < fp->frame_h;
  m.cy = m.cx = 0;
  m.range = fp->me_range;
  m.pr = m.pc = 0;
  m.copy = 0;
  if (level > 0) {
    int pi = ((i / n) >> 1) * (n >> 1) + ((i % n) >> 1);
    const int32_t *par = mv + (sb * NUM_NODES + node_base(level - 1) + pi) * 2;
    m.pr = par[0];
    m.pc = par[1];
    m.cy = m.pr >> 3;
    m.cx = m.pc >> 3;
    m.range = imin(m.range, (fp->turbo & T_ME_CR1) ? 1 : (fp->turbo & T_ME_CR2) ? 2 : 4);
    m.copy = ((fp->turbo & T_ME_L3COPY) || leaf_no8(fp)) && level == 3;
  }
  m.step = 1;
  m.stages = 1;
  if (level == 0) {
    m.step = (fp->turbo & T_ME_HME3) ? 2 * ME_COARSE_STEP : ME_COARSE_STEP;
    m.range = (m.range / m.step) * m.step;
    m.stages = (fp->turbo & T_ME_HME3) ? 3 : 2;
  }
  if (level == 3 && (fp->turbo & T_ME_L3SUB)) m.stages = 0;
  int side = 2 * (m.range / m.step) + 1;
  m.count = 1 + side * side;
  return m;
}

// Later stages of level 0 (k_me.h:182-194).
__device__ void refine_stage(const FrameParams *fp, Node *m, int wy, int wx, int stage) {
  m->cy = wy;
  m->cx = wx;
  if (stage == 1 && (fp->turbo & T_ME_HME3)) {
    m->range = ME_COARSE_STEP;
    m->step = ME_COARSE_STEP;
  } else {
    m->range = (fp->turbo & T_ME_REF2) ? 2 : ME_REFINE;
    m->step = 1;
  }
  int side = 2 * (m->range / m->step) + 1;
  m->count = 1 + side * side;
}

// Candidate k of the current stage: 0 the centre, then the grid in raster order.
__device__ __forceinline__ void candidate(const Node &m, int k, int *dy, int *dx) {
  if (k == 0) {
    *dy = m.cy;
    *dx = m.cx;
    return;
  }
  k -= 1;
  int side = 2 * (m.range / m.step) + 1;
  *dy = m.cy - m.range + (k / side) * m.step;
  *dx = m.cx - m.range + (k % side) * m.step;
}

__device__ __forceinline__ uint32_t load_u32_unaligned(const uint8_t *p) {
  uintptr_t a = (uintptr_t)p;
  const uint32_t *q = (const uint32_t *)(a & ~(uintptr_t)3);
  uint32_t lo = __ldg(q), hi = __ldg(q + 1);
  return __funnelshift_r(lo, hi, (unsigned)(a & 3) * 8);
}

// Full-pel SAD of the w x w block at (x, y) against the reference at offset
// (dy, dx), rows strided by rs, scaled back by rs; reference coordinates
// clamped to the frame (k_me.h:39-64).
__device__ int full_sad(const Frame &f, const Node &m, int dy, int dx, int rs) {
  const FrameParams *fp = f.fp;
  int stride = fp->stride[0], W = fp->frame_w, Hh = fp->frame_h;
  const uint8_t *src = f.src + fp->offset[0], *ref = f.ref + fp->offset[0];
  int w = m.w, x = m.x, y = m.y;
  unsigned sad = 0;
  if (x + dx >= 0 && x + dx + w <= W && y + dy >= 0 && y + dy + w <= Hh) {
    for (int i = 0; i < w; i += rs) {
      const uint32_t *s = (const uint32_t *)(src + (y + i) * stride + x);
      const uint8_t *r = ref + (y + i + dy) * stride + x + dx;
      for (int j = 0; j < (w >> 2); j++) sad = __vsadu4(__ldg(s + j), load_u32_unaligned(r + 4 * j)) + sad;
    }
    return (int)sad * rs;
  }
  for (int i = 0; i < w; i += rs) {
    int ry = clip3(0, Hh - 1, y + i + dy);
    const uint8_t *s = src + (y + i) * stride + x;
    const uint8_t *r = ref + ry * stride;
    for (int j = 0; j < w; j++) sad += iabs((int)s[j] - (int)r[clip3(0, W - 1, x + j + dx)]);
  }
  return (int)sad * rs;
}

// SAD x16 on the decimated planes at offset (dy, dx), multiples of 4 (k_me.h:121-130).
__device__ int dec_sad(const Frame &f, const Node &m, int dy, int dx) {
  const FrameParams *fp = f.fp;
  int W = dec_w(fp), H = dec_h(fp), n = m.w >> 2, x0 = m.x >> 2, y0 = m.y >> 2, oy = dy >> 2, ox = dx >> 2, sad = 0;
  for (int i = 0; i < n; i++) {
    int sy = imin(y0 + i, H - 1), ry = clip3(0, H - 1, y0 + i + oy);
    for (int j = 0; j < n; j++)
      sad += iabs((int)f.dsrc[sy * W + imin(x0 + j, W - 1)] - (int)f.dref[ry * W + clip3(0, W - 1, x0 + j + ox)]);
  }
  return sad * 16;
}

// Full-pel cost (k_me.h:211-220).
__device__ int full_cost(const Frame &f, const Node &m, int dy, int dx) {
  const FrameParams *fp = f.fp;
  int bits = 2 + 2 * floor_log2(iabs(dy) * 8 + 1) + 2 * floor_log2(iabs(dx) * 8 + 1);
  if ((fp->turbo & T_ME_DEC) && m.step >= ME_COARSE_STEP) return dec_sad(f, m, dy, dx) + fp->ac_q[0] * bits / 64;
  int rs = (fp->turbo & T_ME_RSUB) && m.step == 1 ? 2 : 1;
  return full_sad(f, m, dy, dx, rs) + fp->ac_q[0] * bits / 64;
}

// The same cost with the warp's 32 lanes splitting one candidate's byte pairs
// (the 64x64 level: few nodes, so each CTA's four warps take candidates in
// turn instead of one thread a candidate). Every lane returns the total. The
// sums are the ones full_sad / dec_sad form, in another order: unsigned
// integer addition, so the cost is the same.
// Not inlined, with its arguments by value: the kernel's other levels keep
// their registers (inlined, the kernel spills at its 96-register bound).
__device__ __noinline__ int warp_full_cost(const FrameParams *fp, const uint8_t *fsrc, const uint8_t *fref,
                                           const uint8_t *dsrc, const uint8_t *dref, int x, int y, int w, int step,
                                           int dy, int dx, int lane) {
  int bits = 2 + 2 * floor_log2(iabs(dy) * 8 + 1) + 2 * floor_log2(iabs(dx) * 8 + 1);
  unsigned sad = 0;
  int scale;
  if ((fp->turbo & T_ME_DEC) && step >= ME_COARSE_STEP) {
    // dec_sad: n x n pairs of the decimated planes, lanes along rows
    int W = dec_w(fp), H = dec_h(fp), lg = floor_log2(w >> 2), n = 1 << lg;
    int x0 = x >> 2, y0 = y >> 2, oy = dy >> 2, ox = dx >> 2;
    for (int p = lane; p < n * n; p += 32) {
      int i = p >> lg, j = p & (n - 1);
      int sy = imin(y0 + i, H - 1), ry = clip3(0, H - 1, y0 + i + oy);
      sad = __sad((int)dsrc[sy * W + imin(x0 + j, W - 1)], (int)dref[ry * W + clip3(0, W - 1, x0 + j + ox)], sad);
    }
    scale = 16;
  } else {
    // full_sad: rows 0, rs, 2 rs, ... of w / 4 words, lanes along rows
    int rs = (fp->turbo & T_ME_RSUB) && step == 1 ? 2 : 1;
    int stride = fp->stride[0], W = fp->frame_w, Hh = fp->frame_h;
    const uint8_t *src = fsrc + fp->offset[0], *ref = fref + fp->offset[0];
    int lgw = floor_log2(w >> 2), nw = (w / rs) << lgw;
    if (x + dx >= 0 && x + dx + w <= W && y + dy >= 0 && y + dy + w <= Hh) {
      for (int q = lane; q < nw; q += 32) {
        int i = (q >> lgw) * rs, j = q & ((1 << lgw) - 1);
        uint32_t s = __ldg((const uint32_t *)(src + (y + i) * stride + x) + j);
        sad = __vsadu4(s, load_u32_unaligned(ref + (y + i + dy) * stride + x + dx + 4 * j)) + sad;
      }
    } else {
      for (int q = lane; q < nw; q += 32) {
        int i = (q >> lgw) * rs, j = q & ((1 << lgw) - 1);
        const uint8_t *s = src + (y + i) * stride + x + 4 * j;
        const uint8_t *r = ref + clip3(0, Hh - 1, y + i + dy) * stride;
        for (int b = 0; b < 4; b++) sad = __sad((int)s[b], (int)r[clip3(0, W - 1, x + 4 * j + b + dx)], sad);
      }
    }
    scale = rs;
  }
  for (int off = 16; off > 0; off >>= 1) sad += __shfl_xor_sync(0xffffffffu, sad, off);
  return (int)sad * scale + fp->ac_q[0] * bits / 64;
}

// SATD of 4x4 unit u of the node against the quarter-pel plane prediction at
// (mvr, mvc) (even, 1/8 units) (k_me.h:317-340).
__device__ int unit_satd_hp(const Frame &f, const Node &m, int mvr, int mvc, int u) {
  const FrameParams *fp = f.fp;
  int W = fp->frame_w, H = fp->frame_h, nu = m.w >> 2;
  int ux = m.x + (u % nu) * 4, uy = m.y + (u / nu) * 4;
  const uint8_t *pl = f.qp + (size_t)(((mvr >> 1) & 3) * 4 + ((mvc >> 1) & 3)) * W * H;
  int iy = uy + (mvr >> 3), ix = ux + (mvc >> 3);
  const uint8_t *sp = f.src + fp->offset[0] + uy * fp->stride[0] + ux;
  int d[16];
  if (ix >= 0 && ix + 8 <= W && iy >= 0 && iy + 4 <= H) {
    // inside the plane, and the two aligned words each row load stay in the
    // row: no clamping; the source row is word aligned (ux % 4 == 0)
    for (int r = 0; r < 4; r++) {
      uint32_t pv = load_u32_unaligned(pl + (size_t)(iy + r) * W + ix);
      uint32_t sv = __ldg((const uint32_t *)(sp + r * fp->stride[0]));
      for (int c = 0; c < 4; c++) d[r * 4 + c] = (int)((sv >> (8 * c)) & 255) - (int)((pv >> (8 * c)) & 255);
    }
    return pred::satd4x4(d);
  }
  for (int r = 0; r < 4; r++) {
    const uint8_t *row = pl + (size_t)clip3(0, H - 1, iy + r) * W;
    for (int c = 0; c < 4; c++) d[r * 4 + c] = (int)sp[r * fp->stride[0] + c] - (int)row[clip3(0, W - 1, ix + c)];
  }
  return pred::satd4x4(d);
}

// SATD of 4x4 unit u against the normative EIGHTTAP prediction of the node
// at (mvr, mvc) (the non-plane path, k_me.h:254-257).
__device__ int unit_satd_pred(const Frame &f, const Node &m, int mvr, int mvc, int u) {
  const FrameParams *fp = f.fp;
  int nu = m.w >> 2, bx = (u % nu) * 4, by = (u / nu) * 4;
  pred::Inter p;
  pred::inter_setup(&p, f.ref + fp->offset[0], fp->stride[0], fp->frame_w, fp->frame_h, m.x, m.y, m.w, m.w, mvr, mvc,
                    0, 0, EIGHTTAP);
  const uint8_t *sp = f.src + fp->offset[0] + (m.y + by) * fp->stride[0] + m.x + bx;
  int d[16];
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 4; c++) d[r * 4 + c] = (int)sp[r * fp->stride[0] + c] - pred::inter_pixel(&p, by + r, bx + c);
  return pred::satd4x4(d);
}

__device__ __forceinline__ void sub_neighbour(const FrameParams *fp, int j, int step, int *dr, int *dc) {
  int k = (fp->turbo & T_ME_CROSS) ? (j == 0 ? 1 : j == 1 ? 3 : j == 2 ? 4 : 6) : j;
  *dr = (k < 3) ? -step : (k < 5 ? 0 : step);
  *dc = (k == 0 || k == 3 || k == 5) ? -step : ((k == 1 || k == 6) ? 0 : step);
}

// The threads searching one node: the CTA (the 64x64 level), a warp, or
// half a warp (the 8x8 level, whose nodes have at most 16 sub-pel pairs at
// a time); mask holds the group's lanes of its warp.
struct MeGrp {
  int rank, size;
  unsigned mask;
  __device__ __forceinline__ void sync() const {
    if (size > 32) __syncthreads();
    else __syncwarp(mask);
  }
};

// Minimum over the group's lanes of its warp (the whole warp for a CTA group).
__device__ __forceinline__ unsigned long long group_min(unsigned long long v, const MeGrp &g) {
  for (int off = g.size >= 32 ? 16 : g.size >> 1; off > 0; off >>= 1) {
    unsigned long long o = __shfl_xor_sync(g.mask, v, off);
    v = o < v ? o : v;
  }
  return v;
}

// Sub-pel costs of ncand candidates (mvr[c], mvc[c]) into cost[c] (shared,
// private to the group), every (candidate, unit) pair spread over the group.
__device__ void subpel_costs(const Frame &f, const Node &m, const int *cr, const int *cc, int ncand, int *cost,
                             const MeGrp &g) {
  const FrameParams *fp = f.fp;
  int hp = (fp->turbo & T_ME_HPEL) != 0;
  int nu = (m.w >> 2) * (m.w >> 2);
  int st = hp && (fp->turbo & T_ME_USUB) && m.w >= 32 ? 2 : 1;
  int nus = (nu + st - 1) / st;
  if (g.rank < ncand) cost[g.rank] = 0;
  if (g.rank == 0) WORK(W_ME_SATD, ncand * nus);
  g.sync();
  for (int p = g.rank; p < ncand * nus; p += g.size) {
    int c = p / nus, u = (p % nus) * st;
    int s = hp ? unit_satd_hp(f, m, cr[c], cc[c], u) : unit_satd_pred(f, m, cr[c], cc[c], u);
    atomicAdd(&cost[c], s);
  }
  g.sync();
  if (g.rank < ncand) cost[g.rank] *= st;
  g.sync();
}

// One search level: with group 128 the CTA's four warps per node (the 64x64
// level: few, large nodes), with 32 a warp per (node, reference), with 16
// half a warp (the 8x8 level); blockIdx.y selects the reference.
// At least 5 CTAs per SM (at most 102 registers a thread): more resident
// warps hide the L2 latency of the candidates' SAD rows (measured on the
// 1080p clip: an ALTREF frame's search 0.46 -> 0.36 ms; 8 CTAs spill).
#ifndef MAV1CU_ME_MIN_CTAS
#define MAV1CU_ME_MIN_CTAS 5
#endif
__global__ void __launch_bounds__(128, MAV1CU_ME_MIN_CTAS) k_me_level(Frame f0, Frame f1, int level, int group) {
  __shared__ int s_cost[8][16];
  __shared__ int s_r[8][16], s_c[8][16];
  __shared__ unsigned long long s_best[4];
  const Frame &f = blockIdx.y ? f1 : f0;
  const FrameParams *fp = f.fp;
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int whole_cta = group == 128, half = lane >> 4;
  MeGrp grp = whole_cta ? MeGrp{(int)threadIdx.x, 128, 0xffffffffu}
              : group == 32 ? MeGrp{lane, 32, 0xffffffffu}
                            : MeGrp{lane & 15, 16, 0xffffu << (16 * half)};
  int slotw = whole_cta ? 0 : group == 32 ? warp : 2 * warp + half;
  int nn = 1 << (2 * level);
  int g = whole_cta ? (int)blockIdx.x : (int)blockIdx.x * (128 / group) + slotw;
  if (g >= fp->sb_cols * fp->sb_rows * nn) return;
  int sb = g / nn, i = g % nn;
  Node m = make_node(fp, sb, level, i, f.mv);
  if (f.isGold && level == 3 && (fp->turbo & T_ME_G3COPY) && fp->leaf && !fp->frame_is_intra) m.copy = 1;
  int32_t *out = f.mv + (sb * NUM_NODES + node_base(level) + i) * 2;
  if (!m.valid) {
    if (grp.rank == 0) out[0] = out[1] = 0;
    return;
  }
  if (m.copy) {
    if (grp.rank == 0) {
      out[0] = m.pr;
      out[1] = m.pc;
    }
    return;
  }
  int by = 0, bx = 0;
  for (int stage = 0; stage < m.stages; stage++) {
    if (stage > 0) refine_stage(fp, &m, by, bx, stage);
    if (grp.rank == 0) {  // byte pairs of the stage's candidates (full_cost)
      int dec = (fp->turbo & T_ME_DEC) && m.step >= ME_COARSE_STEP, rs = (fp->turbo & T_ME_RSUB) && m.step == 1 ? 2 : 1;
      WORK(dec ? W_ME_DSAD : W_ME_SAD, (long long)m.count * (dec ? (m.w >> 2) * (m.w >> 2) : (m.w / rs) * m.w));
    }
    unsigned long long best = ~0ull;
    if (whole_cta) {
      // a warp per candidate, every lane holding the warp's running minimum
      for (int k = warp; k < m.count; k += 4) {
        int dy, dx;
        candidate(m, k, &dy, &dx);
        int cost = warp_full_cost(fp, f.src, f.ref, f.dsrc, f.dref, m.x, m.y, m.w, m.step, dy, dx, lane);
        unsigned long long key = ((unsigned long long)(unsigned)cost << 32) | (unsigned)k;
        best = key < best ? key : best;
      }
    } else {
      for (int k = grp.rank; k < m.count; k += grp.size) {
        int dy, dx;
        candidate(m, k, &dy, &dx);
        unsigned long long key = ((unsigned long long)(unsigned)full_cost(f, m, dy, dx) << 32) | (unsigned)k;
        best = key < best ? key : best;
      }
    }
    best = group_min(best, grp);
    if (whole_cta) {
      __syncthreads();
      if (lane == 0) s_best[warp] = best;
      __syncthreads();
      for (int w = 0; w < 4; w++) best = s_best[w] < best ? s_best[w] : best;
    }
    candidate(m, (int)(best & 0xffffffffu), &by, &bx);
  }
  if (level > 0 && (m.copy || ((fp->turbo & T_ME_KEEP) && by == m.cy && bx == m.cx))) {
    if (grp.rank == 0) {
      out[0] = m.pr;
      out[1] = m.pc;
    }
    return;
  }
  // sub-pel refinement (k_me.h:262-281)
  int *cost = s_cost[slotw], *cr = s_r[slotw], *cc = s_c[slotw];
  int mvr = m.stages ? by * 8 : m.pr, mvc = m.stages ? bx * 8 : m.pc;
  if (grp.rank == 0) {
    cr[0] = mvr;
    cc[0] = mvc;
  }
  grp.sync();
  subpel_costs(f, m, cr, cc, 1, cost, grp);
  int bestS = cost[0];
  int minStep = m.w >= 32 && (fp->turbo & T_ME_HALF01) ? 4 : 2;
  int nb = (fp->turbo & T_ME_CROSS) ? 4 : 8;
  for (int step = 4; step >= minStep; step >>= 1) {
    grp.sync();
    if (grp.rank < nb) {
      int dr, dc;
      sub_neighbour(fp, grp.rank, step, &dr, &dc);
      cr[grp.rank] = mvr + dr;
      cc[grp.rank] = mvc + dc;
    }
    grp.sync();
    subpel_costs(f, m, cr, cc, nb, cost, grp);
    // running strict minimum over the neighbours in order == first minimum
    int bk = -1, bc = bestS;
    for (int k = 0; k < nb; k++)
      if (cost[k] < bc) {
        bc = cost[k];
        bk = k;
      }
    if (bk >= 0) {
      bestS = bc;
      mvr = cr[bk];
      mvc = cc[bk];
    }
  }
  if (grp.rank == 0) {
    out[0] = mvr;
    out[1] = mvc;
  }
}

}  // namespace me
