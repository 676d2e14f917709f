// Loop-restoration parameter search on the device: the reference's lr_select
// (src/lr_search.c:244-359) with its Wiener least-squares fit (wiener_fit,
// :142-193), its self-guided projection fit (sgr_fit, :196-240), the unit SSE
// (unit_sse, :92-108) and the rate of the unit parameters (lr_unit_params /
// lr_subexp, :33-80).
//
// Per restoration unit the reference compares RESTORE_NONE, a fitted Wiener
// filter refined greedily by +-1 tap steps, and every self-guided set with
// fitted projection weights, by 16 * SSE + lambda * bits. The rate of a unit's
// parameters depends on the parameters the previous unit of the plane chose
// (subexponential coding against running references), so the choice is a
// serial scan over the units. Everything that does not depend on those
// references is computed first, for all units at once:
//
//   k_lr_fit     one CTA per unit: the SSE of RESTORE_NONE, the Wiener fit,
//                the SSE of the fitted filter and of its single-tap
//                neighbours (the candidates the refinement tries first), and
//                per self-guided set the fit and its SSE;
//   k_lr_spec    one CTA per unit: the Wiener refinement replayed under
//                guessed running references, caching the SSE of every
//                candidate it visits (SSEs do not depend on the references);
//   k_lr_select  one CTA per plane, units in order: the rate comparisons of
//                lr_select with the running references; a refinement
//                candidate whose SSE neither pass cached is evaluated on the
//                spot by the whole CTA.
//
// Bit-exactness. SSEs, the self-guided sums and the first Wiener iteration
// are integer-valued (every partial sum is an integer below 2^53, so double
// and int64 sums agree in any order). The later Wiener iterations accumulate
// non-integer doubles: they are summed in the reference's order (the unit's
// 4x4 blocks in raster order, each block's samples in raster order) by one
// lane per accumulator, and every double operation is the reference's, in
// its order, with explicit round-to-nearest intrinsics (no contraction into
// fused multiply-adds). lround is restated as round-half-away-from-zero.
#pragma once

#include "common.cuh"
#include "filters.cuh"

namespace lrs {

using flt::LrBlock;
using flt::lr_block_setup;
using flt::lr_src;

constexpr int THREADS = 256;
constexpr int CACHE = 40;       // candidate SSEs a unit keeps from the first pass and the speculative pass
constexpr int ROWBUF = 4 * 96;  // samples of one block row of a unit (4 rows of at most 95)

// What the first pass leaves for the serial choice, per unit.
struct Fit {
  long long sse_none;
  int w[2][3];                  // fitted Wiener taps
  int n;                        // cached Wiener candidates
  int taps[CACHE][6];           // their taps: pass 0 j 0..2, pass 1 j 0..2
  long long sse[CACHE];
  int xqd[16][2];               // fitted projection weights per self-guided set
  long long sgr_sse[16];
};

// The unit's 4x4 luma block range: rows [r0, r1), columns [c0, c1) of the
// frame's 4x4 grid whose blocks lr_block_setup assigns to unit (ur, uc) of
// the plane (the counting sort of lr_select, lr_search.c:250-272, keeps them
// in raster order).
struct Geom {
  int plane, ur, uc, r0, r1, c0, c1;
};

HD int unit_row_of(const FrameParams *fp, int plane, int r) {
  return imin(fp->lr_unit_rows[plane] - 1, ((r * MI_SIZE + 8) >> (plane > 0)) / fp->lr_unit_size[plane]);
}
HD int unit_col_of(const FrameParams *fp, int plane, int c) {
  return imin(fp->lr_unit_cols[plane] - 1, ((c * MI_SIZE) >> (plane > 0)) / fp->lr_unit_size[plane]);
}

// First r in [0, n) with of(r) >= v, or n: unit_row_of / unit_col_of are
// non-decreasing in r (a clamped quotient of a growing numerator).
template <typename F>
__device__ __forceinline__ int first_at_least(int n, int v, F of) {
  int lo = 0, hi = n;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (of(mid) >= v) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

// The 4x4 rows and columns whose unit is (ur, uc): the contiguous run of r
// with unit_row_of(r) == ur (and the same for columns), found by binary
// search since the maps are non-decreasing; an empty run leaves
// r0 = rows4, r1 = 0 (c0 = cols4, c1 = 0).
__device__ void unit_geom(const FrameParams *fp, int plane, int ur, int uc, Geom *g) {
  int rows4 = (fp->frame_h + 3) >> 2, cols4 = (fp->frame_w + 3) >> 2;
  g->plane = plane;
  g->ur = ur;
  g->uc = uc;
  auto rowOf = [&](int r) { return unit_row_of(fp, plane, r); };
  auto colOf = [&](int c) { return unit_col_of(fp, plane, c); };
  int r0 = first_at_least(rows4, ur, rowOf), r1 = first_at_least(rows4, ur + 1, rowOf);
  int c0 = first_at_least(cols4, uc, colOf), c1 = first_at_least(cols4, uc + 1, colOf);
  g->r0 = r0 < r1 ? r0 : rows4;
  g->r1 = r0 < r1 ? r1 : 0;
  g->c0 = c0 < c1 ? c0 : cols4;
  g->c1 = c0 < c1 ? c1 : 0;
}

// A unit's samples staged in shared memory: the CDEF output, the deblocked
// frame and the source over the unit plus 3 samples on every side (clamped to
// the plane), which covers every tap the filters read for the unit's blocks
// (get_source_sample moves a row at most to the block's own 3-row margin).
// A unit spans at most 103 x 95 samples (the last unit row or column takes
// the remainder, and unit rows are offset by 8 luma rows).
constexpr int WP = 104, WH = 112;

struct Win {
  uint8_t cd[WH * WP], db[WH * WP], sr[WH * WP];
  int x0, y0;
};

struct WinSrc {
  const Win *w;
  HD int tap(const LrBlock *lb, int x, int y) const {
    x = imax(0, imin(lb->planeEndX, x));
    y = imax(0, imin(lb->planeEndY, y));
    const uint8_t *b = w->cd;
    if (y < lb->stripeStart) {
      y = imax(lb->stripeStart - 2, y);
      b = w->db;
    } else if (y > lb->stripeEnd) {
      y = imin(lb->stripeEnd + 2, y);
      b = w->db;
    }
    return b[(y - w->y0) * WP + (x - w->x0)];
  }
  HD int own(int x, int y) const { return w->cd[(y - w->y0) * WP + (x - w->x0)]; }
  HD int src(int x, int y) const { return w->sr[(y - w->y0) * WP + (x - w->x0)]; }
};

// Copies the unit's window into shared memory (the whole CTA).
__device__ void stage_window(const FrameParams *fp, const Geom &g, const uint8_t *cdef, const uint8_t *dbk,
                             const uint8_t *src, Win &w) {
  const int sub = g.plane > 0, bw = MI_SIZE >> sub;
  const int endX = ((fp->frame_w + sub) >> sub) - 1, endY = ((fp->frame_h + sub) >> sub) - 1;
  const int x0 = imax(0, ((g.c0 * MI_SIZE) >> sub) - 3), y0 = imax(0, ((g.r0 * MI_SIZE) >> sub) - 3);
  const int x1 = imin(endX, ((g.c1 - 1) * MI_SIZE >> sub) + bw - 1 + 3);
  const int y1 = imin(endY, ((g.r1 - 1) * MI_SIZE >> sub) + bw - 1 + 3);
  const int nx = imin(WP, x1 - x0 + 1), ny = imin(WH, y1 - y0 + 1);
  const int stride = fp->stride[g.plane], off = fp->offset[g.plane];
  if (threadIdx.x == 0) {
    w.x0 = x0;
    w.y0 = y0;
  }
  for (int i = threadIdx.x; i < nx * ny; i += blockDim.x) {
    int r = i / nx, c = i - r * nx;
    int o = off + (y0 + r) * stride + x0 + c, k = r * WP + c;
    w.cd[k] = cdef[o];
    w.db[k] = dbk[o];
    w.sr[k] = src[o];
  }
  __syncthreads();
}

// ---- double arithmetic exactly as the reference's C (no contraction) ---------
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }
// C lround: the nearest integer, halfway cases away from zero.
__device__ __forceinline__ long long lround_away(double x) {
  double t = trunc(x);
  if (fabs(dsub(x, t)) >= 0.5) t = dadd(t, x < 0 ? -1.0 : 1.0);
  return (long long)t;
}

// Gaussian elimination with partial pivoting (solve, lr_search.c:111-138).
__device__ int solve(int n, double M[3][3], double v[3], double *x) {
  for (int i = 0; i < n; i++) {
    int p = i;
    for (int r = i + 1; r < n; r++)
      if (fabs(M[r][i]) > fabs(M[p][i])) p = r;
    if (fabs(M[p][i]) < 1e-9) return 0;
    if (p != i) {
      for (int k = 0; k < n; k++) {
        double t = M[i][k];
        M[i][k] = M[p][k];
        M[p][k] = t;
      }
      double t = v[i];
      v[i] = v[p];
      v[p] = t;
    }
    for (int r = i + 1; r < n; r++) {
      double f = ddiv(M[r][i], M[i][i]);
      for (int k = i; k < n; k++) M[r][k] = dsub(M[r][k], dmul(f, M[i][k]));
      v[r] = dsub(v[r], dmul(f, v[i]));
    }
  }
  for (int i = n - 1; i >= 0; i--) {
    double s = v[i];
    for (int k = i + 1; k < n; k++) s = dsub(s, dmul(M[i][k], x[k]));
    x[i] = ddiv(s, M[i][i]);
  }
  return 1;
}

// ---- rate of the unit parameters (lr_subexp / lr_unit_params) -------------------
HD int recenter_nonneg(int r, int v) {
  if (v > (r << 1)) return v;
  if (v >= r) return (v - r) << 1;
  return ((r - v) << 1) - 1;
}

// bits of v coded as decode_signed_subexp_with_ref_bool( low, high, k, r )
HD int subexp_bits(int low, int high, int k, int r, int v) {
  int mx = high - low;
  r -= low;
  v -= low;
  int x = (r << 1) <= mx ? recenter_nonneg(r, v) : recenter_nonneg(mx - 1 - r, mx - 1 - v);
  int bits = 0, i = 0, mk = 0;
  for (;;) {
    int b2 = i ? k + i - 1 : k;
    int a = 1 << b2;
    if (mx <= mk + 3 * a) {
      int n = mx - mk, val = x - mk;
      int w = floor_log2(n) + 1, m = (1 << w) - n;
      if (val < m) return bits + (w - 1);
      return bits + (w - 1) + 1;
    }
    int more = x >= mk + a;
    bits += 1;
    if (!more) return bits + b2;
    i++;
    mk += a;
  }
}

// Bits of a unit's parameters against the running references, which it then
// takes (read_lr_unit's order).
HD int unit_bits(int plane, const LrUnit &u, int refW[2][3], int refX[2]) {
  int bits = 0;
  if (u.type == RESTORE_WIENER) {
    for (int pass = 0; pass < 2; pass++)
      for (int j = plane ? 1 : 0; j < 3; j++) {
        bits += subexp_bits(T(Wiener_Taps_Min)[j], T(Wiener_Taps_Max)[j] + 1, T(Wiener_Taps_K)[j], refW[pass][j],
                            u.wiener[pass][j]);
        refW[pass][j] = u.wiener[pass][j];
      }
  } else if (u.type == RESTORE_SGRPROJ) {
    bits += 4;  // SGRPROJ_PARAMS_BITS
    for (int i = 0; i < 2; i++) {
      if (T(Sgr_Params)[u.set][i * 2])
        bits += subexp_bits(T(Sgrproj_Xqd_Min)[i], T(Sgrproj_Xqd_Max)[i] + 1, 4 /* SGRPROJ_PRJ_SUBEXP_K */, refX[i],
                            u.xqd[i]);
      refX[i] = u.xqd[i];
    }
  }
  return bits;
}

HD long long rd(const FrameParams *fp, long long sse, int bits) { return sse * 16 + (long long)fp->lambda * bits; }

// ---- CTA-wide helpers ------------------------------------------------------------------
struct Shared {
  Win win;
  double phi[2][ROWBUF][4];  // per sample of a block row: phi[0..nc) and the target
  double acc[12];
  double f[7], g[7];
  long long red[THREADS / 32];
  Geom geom;
  int stop;
  // k_lr_spec: the unit's candidate cache (Fit::taps / sse / n), kept by thread 0
  int ctaps[CACHE][6];
  long long csse[CACHE];
  int cn;
  // k_lr_select: the unit's first-pass results, and a cache lookup's result
  Fit fit;
  int found;
};

// Sum of v over the CTA (every thread gets it).
__device__ long long cta_sum(long long v, Shared &sh) {
  for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh.red[threadIdx.x >> 5] = v;
  __syncthreads();
  long long s = 0;
  for (int w = 0; w < THREADS / 32; w++) s += sh.red[w];
  __syncthreads();
  return s;
}

struct SseSink {
  const Win *w;
  long long sse;
  HD void operator()(int x, int y, int v) {
    int d = v - (int)w->sr[(y - w->y0) * WP + (x - w->x0)];
    sse += d * d;
  }
};

// SSE of a unit filtered with u against the source (unit_sse), from the
// staged window: a thread per 4x4 block of the unit.
__device__ long long unit_sse(const FrameParams *fp, const Geom &g, const LrUnit &u, Shared &sh) {
  int nc = g.c1 - g.c0, nb = (g.r1 - g.r0) * nc;
  WinSrc in{&sh.win};
  SseSink sink{&sh.win, 0};
  for (int b = threadIdx.x; b < nb; b += THREADS) {
    LrBlock lb;
    if (!lr_block_setup(fp, g.plane, g.r0 + b / nc, g.c0 + b % nc, &lb)) continue;
    if (u.type == RESTORE_WIENER) {
      flt::lr_wiener_to(&lb, in, &u, sink);
    } else if (u.type == RESTORE_SGRPROJ) {
      int flt0[16], flt1[16];
      flt::lr_box(&lb, in, u.set, 0, flt0);
      flt::lr_box(&lb, in, u.set, 1, flt1);
      flt::lr_sgr_project(&lb, in, &u, flt0, flt1, sink);
    } else {
      for (int i = 0; i < lb.h; i++)
        for (int j = 0; j < lb.w; j++) sink(lb.x + j, lb.y + i, in.own(lb.x + j, lb.y + i));
    }
  }
  return cta_sum(sink.sse, sh);
}

HD LrUnit wiener_unit(const int w[2][3]) {
  LrUnit u = {};
  u.type = RESTORE_WIENER;
  for (int p = 0; p < 2; p++)
    for (int j = 0; j < 3; j++) u.wiener[p][j] = w[p][j];
  return u;
}

// wiener_fit (lr_search.c:142-193): four alternating separable least-squares
// solves, then the taps in coded units.
__device__ void wiener_fit(const FrameParams *fp, const Geom &g, Shared &sh, int out[2][3]) {
  const int plane = g.plane, first = plane ? 1 : 0, nc = 3 - first, nacc = nc * nc + nc;
  const int sub = plane > 0, bwf = MI_SIZE >> sub;
  const WinSrc in{&sh.win};
  if (threadIdx.x < 7) {
    sh.f[threadIdx.x] = threadIdx.x == 3 ? 1.0 : 0.0;
    sh.g[threadIdx.x] = threadIdx.x == 3 ? 1.0 : 0.0;
  }
  if (threadIdx.x == 0) sh.stop = 0;
  __syncthreads();
  for (int iter = 0; iter < 4 && !sh.stop; iter++) {
    const int vertical = !(iter & 1);
    double acc = 0.0;  // lane L < nacc of warp 0: M[L / nc][L % nc], then V[L - nc * nc]
    for (int r = g.r0; r < g.r1; r++) {
      // the block row's samples in the reference's order: blocks left to
      // right, each block's rows, each row's samples
      LrBlock lb0;
      lr_block_setup(fp, plane, r, g.c0, &lb0);
      const int h = lb0.h;
      int wsum = 0;
      for (int c = g.c0; c < g.c1; c++) wsum += imin(bwf, lb0.planeEndX - ((c * MI_SIZE) >> sub) + 1);
      const int npx = h * wsum;
      const int buf = r & 1;
      for (int k = threadIdx.x; k < npx; k += THREADS) {
        // k -> (block column, row, column): full blocks are bwf wide, only the
        // plane's last column of blocks can be narrower
        int cb = k / (bwf * h);
        int rem = k - cb * bwf * h;
        LrBlock lb;
        lr_block_setup(fp, plane, r, g.c0 + cb, &lb);
        int i = rem / lb.w, j = rem - i * lb.w;
        double Z[7];
        for (int kk = 0; kk < 7; kk++) {
          double s = 0.0;
          for (int t = 0; t < 7; t++) {
            int sv = vertical ? in.tap(&lb, lb.x + j + t - 3, lb.y + i + kk - 3)
                              : in.tap(&lb, lb.x + j + kk - 3, lb.y + i + t - 3);
            s = dadd(s, dmul(vertical ? sh.g[t] : sh.f[t], (double)sv));
          }
          Z[kk] = s;
        }
        for (int kk = first; kk < 3; kk++) sh.phi[buf][k][kk - first] = dsub(dadd(Z[kk], Z[6 - kk]), dmul(2.0, Z[3]));
        sh.phi[buf][k][3] = dsub((double)in.src(lb.x + j, lb.y + i), Z[3]);
      }
      __syncthreads();
      if (threadIdx.x < nacc) {
        int L = threadIdx.x;
        int a = L < nc * nc ? L / nc : L - nc * nc;
        int b = L < nc * nc ? L % nc : 3;
        for (int k = 0; k < npx; k++) acc = dadd(acc, dmul(sh.phi[buf][k][a], sh.phi[buf][k][b]));
      }
      // the next row writes the other buffer; this one is read until the
      // barrier after that row's samples
    }
    if (threadIdx.x < nacc) sh.acc[threadIdx.x] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double M[3][3] = {{0}}, V[3] = {0}, x[3] = {0, 0, 0};
      for (int a = 0; a < nc; a++) {
        for (int b = 0; b < nc; b++) M[a][b] = sh.acc[a * nc + b];
        V[a] = sh.acc[nc * nc + a];
      }
      for (int a = 0; a < nc; a++) M[a][a] = dadd(M[a][a], 1e-3);
      if (!solve(nc, M, V, x)) {
        sh.stop = 1;
      } else {
        double *dst = vertical ? sh.f : sh.g;
        double sum = 0.0;
        for (int k = 0; k < 3; k++) {
          double v = k < first ? 0.0 : x[k - first];
          dst[k] = dst[6 - k] = v;
          sum = dadd(sum, v);
        }
        dst[3] = dsub(1.0, dmul(2.0, sum));
      }
    }
    __syncthreads();
  }
  for (int pass = 0; pass < 2; pass++) {
    const double *sv = pass == 0 ? sh.f : sh.g;
    for (int j = 0; j < 3; j++) {
      int v = j < first ? 0 : (int)lround_away(dmul(sv[j], 128.0));
      out[pass][j] = j < first ? 0 : imax(T(Wiener_Taps_Min)[j], imin(T(Wiener_Taps_Max)[j], v));
    }
  }
  __syncthreads();
}

// sgr_fit (lr_search.c:196-240): least-squares projection weights of set
// `set`. The sums are integer-valued and exact in int64; the closing double
// arithmetic follows the reference's operations.
__device__ void sgr_fit(const FrameParams *fp, const Geom &g, int set, Shared &sh, int xqd[2]) {
  const int r0 = T(Sgr_Params)[set][0], r1 = T(Sgr_Params)[set][2];
  const int ncols = g.c1 - g.c0, nb = (g.r1 - g.r0) * ncols;
  const WinSrc in{&sh.win};
  long long h00 = 0, h01 = 0, h11 = 0, c0 = 0, c1 = 0;
  for (int b = threadIdx.x; b < nb; b += THREADS) {
    LrBlock lb;
    if (!lr_block_setup(fp, g.plane, g.r0 + b / ncols, g.c0 + b % ncols, &lb)) continue;
    int flt0[16], flt1[16];
    flt::lr_box(&lb, in, set, 0, flt0);
    flt::lr_box(&lb, in, set, 1, flt1);
    for (int i = 0; i < lb.h; i++)
      for (int j = 0; j < lb.w; j++) {
        long long u = (long long)in.own(lb.x + j, lb.y + i) << SGRPROJ_RST_BITS;
        long long s = ((long long)in.src(lb.x + j, lb.y + i) << SGRPROJ_RST_BITS) - u;
        long long f0 = r0 ? flt0[i * 4 + j] - u : 0, f1 = r1 ? flt1[i * 4 + j] - u : 0;
        h00 += f0 * f0;
        h01 += f0 * f1;
        h11 += f1 * f1;
        c0 += f0 * s;
        c1 += f1 * s;
      }
  }
  double H00 = (double)cta_sum(h00, sh), H01 = (double)cta_sum(h01, sh), H11 = (double)cta_sum(h11, sh);
  double C0 = (double)cta_sum(c0, sh), C1 = (double)cta_sum(c1, sh);
  double a = 0.0, bb = 0.0;
  if (r0 && r1) {
    double det = dsub(dmul(H00, H11), dmul(H01, H01));
    if (fabs(det) > 1e-9) {
      a = ddiv(dsub(dmul(C0, H11), dmul(C1, H01)), det);
      bb = ddiv(dsub(dmul(C1, H00), dmul(C0, H01)), det);
    }
  } else if (r0) {
    if (H00 > 0) a = ddiv(C0, H00);
  } else if (r1) {
    if (H11 > 0) bb = ddiv(C1, H11);
  }
  int w0 = (int)lround_away(dmul(a, (double)(1 << SGRPROJ_PRJ_BITS)));
  int w2 = (int)lround_away(dmul(bb, (double)(1 << SGRPROJ_PRJ_BITS)));
  if (!r0) w0 = 0;
  xqd[0] = imax(T(Sgrproj_Xqd_Min)[0], imin(T(Sgrproj_Xqd_Max)[0], w0));
  if (!r1)
    xqd[1] = imax(T(Sgrproj_Xqd_Min)[1], imin(T(Sgrproj_Xqd_Max)[1], (1 << SGRPROJ_PRJ_BITS) - xqd[0]));
  else
    xqd[1] = imax(T(Sgrproj_Xqd_Min)[1], imin(T(Sgrproj_Xqd_Max)[1], (1 << SGRPROJ_PRJ_BITS) - xqd[0] - w2));
}

HD void taps_of(const LrUnit &u, int *t) {
  for (int p = 0; p < 2; p++)
    for (int j = 0; j < 3; j++) t[p * 3 + j] = u.wiener[p][j];
}

// First pass: one CTA per unit (all planes; the unit's index in LRUNITS).
__global__ void __launch_bounds__(THREADS) k_lr_fit(const FrameParams *fp, const uint8_t *cdef, const uint8_t *dbk,
                                                   const uint8_t *src, Fit *fits) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Shared &sh = *reinterpret_cast<Shared *>(smem_raw);
  const int gu = blockIdx.x;
  int plane = 2;
  while (plane > 0 && gu < fp->lr_unit_off[plane]) plane--;
  const int u = gu - fp->lr_unit_off[plane];
  if (threadIdx.x == 0) unit_geom(fp, plane, u / fp->lr_unit_cols[plane], u % fp->lr_unit_cols[plane], &sh.geom);
  __syncthreads();
  const Geom g = sh.geom;
  stage_window(fp, g, cdef, dbk, src, sh.win);
  Fit &F = fits[gu];
  LrUnit none = {};
  none.type = RESTORE_NONE;
  long long sseNone = unit_sse(fp, g, none, sh);
  int w[2][3];
  wiener_fit(fp, g, sh, w);
  // the fitted filter and its single-tap neighbours, in the refinement's order
  int n = 0;
  LrUnit base = wiener_unit(w);
  long long sseW = unit_sse(fp, g, base, sh);
  if (threadIdx.x == 0) {
    taps_of(base, F.taps[n]);
    F.sse[n] = sseW;
  }
  n++;
  for (int pass = 0; pass < 2; pass++)
    for (int j = plane ? 1 : 0; j < 3; j++)
      for (int d = -1; d <= 1; d += 2) {
        LrUnit t = base;
        t.wiener[pass][j] += d;
        if (t.wiener[pass][j] < T(Wiener_Taps_Min)[j] || t.wiener[pass][j] > T(Wiener_Taps_Max)[j]) continue;
        long long sse = unit_sse(fp, g, t, sh);
        if (threadIdx.x == 0) {
          taps_of(t, F.taps[n]);
          F.sse[n] = sse;
        }
        n++;
      }
  for (int set = 0; set < 16; set++) {
    int xqd[2];
    sgr_fit(fp, g, set, sh, xqd);
    LrUnit s = {};
    s.type = RESTORE_SGRPROJ;
    s.set = set;
    s.xqd[0] = xqd[0];
    s.xqd[1] = xqd[1];
    long long sse = unit_sse(fp, g, s, sh);
    if (threadIdx.x == 0) {
      F.xqd[set][0] = xqd[0];
      F.xqd[set][1] = xqd[1];
      F.sgr_sse[set] = sse;
    }
  }
  if (threadIdx.x == 0) {
    F.sse_none = sseNone;
    F.n = n;
    for (int p = 0; p < 2; p++)
      for (int j = 0; j < 3; j++) F.w[p][j] = w[p][j];
  }
}

// SSE of Wiener candidate t: the first pass's value when it has one, else
// computed by the whole CTA from the unit's window, staged at the first such
// candidate of the unit (every thread calls this with the same t).
// Index of the cache entry holding taps tt (entries are distinct), or -1:
// thread i compares entry i (the whole CTA).
__device__ int cache_find(const int (*taps)[6], int n, const int *tt, Shared &sh) {
  if (threadIdx.x == 0) sh.found = -1;
  __syncthreads();
  int i = threadIdx.x;
  if (i < n) {
    bool eq = true;
    for (int k = 0; k < 6; k++) eq = eq && taps[i][k] == tt[k];
    if (eq) sh.found = i;
  }
  __syncthreads();
  int f = sh.found;
  __syncthreads();
  return f;
}

__device__ long long wiener_sse(const FrameParams *fp, const Fit &F, const Geom &g, const uint8_t *cdef,
                                const uint8_t *dbk, const uint8_t *src, const LrUnit &t, Shared &sh, bool &staged) {
  int tt[6];
  taps_of(t, tt);
  int f = cache_find(F.taps, F.n, tt, sh);
  if (f >= 0) return F.sse[f];
  if (!staged) {
    stage_window(fp, g, cdef, dbk, src, sh.win);
    staged = true;
  }
  return unit_sse(fp, g, t, sh);
}

// Second pass: one CTA per plane, the units in order (lr_select's loop,
// lr_search.c:276-355). Every thread runs the same scalar decisions; the SSE
// of a candidate the first pass did not compute is evaluated by all of them.
// Speculative refinement, one CTA per unit, after k_lr_fit: the Wiener
// refinement of lr_select (lr_search.c:296-318) replayed for the unit under
// guessed running references, computing and caching the SSE of every
// candidate the cache does not hold yet. An SSE depends on the candidate
// filter and the unit's samples only, never on the references, so a cached
// value is exactly what the serial choice would compute; the references only
// decide which candidates the refinement visits. The guesses: the default
// references (exact for a plane's first unit) and the fitted filter of each
// of the two previous units (the true reference is usually the refined
// filter of a recent unit). k_lr_select then finds most of its candidates
// here and computes only the rest on the spot.
__device__ void spec_path(const FrameParams *fp, int plane, const Geom &g, const uint8_t *cdef, const uint8_t *dbk,
                          const uint8_t *src, const int fitted[2][3], const int ref[2][3], Shared &sh, bool &staged) {
  LrUnit w = wiener_unit(fitted);
  int tw[2][3], tx[2] = {0, 0};
  memcpy(tw, ref, sizeof tw);
  long long wc = rd(fp, sh.csse[0], 2 + unit_bits(plane, w, tw, tx));
  for (int pass = 0; pass < 2; pass++)
    for (int j = plane ? 1 : 0; j < 3; j++)
      for (int d = -1; d <= 1; d += 2) {
        LrUnit t = w;
        t.wiener[pass][j] += d;
        if (t.wiener[pass][j] < T(Wiener_Taps_Min)[j] || t.wiener[pass][j] > T(Wiener_Taps_Max)[j]) continue;
        int tt[6];
        taps_of(t, tt);
        int n = sh.cn;
        int f = cache_find(sh.ctaps, n, tt, sh);
        long long sse = f >= 0 ? sh.csse[f] : -1;
        if (sse < 0) {
          if (n >= CACHE) return;  // full: the serial choice computes the rest
          if (!staged) {
            stage_window(fp, g, cdef, dbk, src, sh.win);
            staged = true;
          }
          sse = unit_sse(fp, g, t, sh);  // the whole CTA; every thread gets the sum
          if (threadIdx.x == 0) {
            for (int k = 0; k < 6; k++) sh.ctaps[n][k] = tt[k];
            sh.csse[n] = sse;
            sh.cn = n + 1;
          }
          __syncthreads();
        }
        memcpy(tw, ref, sizeof tw);
        long long tc = rd(fp, sse, 2 + unit_bits(plane, t, tw, tx));
        if (tc < wc) {
          wc = tc;
          w = t;
        }
      }
}

__global__ void __launch_bounds__(THREADS) k_lr_spec(const FrameParams *fp, const uint8_t *cdef, const uint8_t *dbk,
                                                    const uint8_t *src, Fit *fits) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Shared &sh = *reinterpret_cast<Shared *>(smem_raw);
  const int gu = blockIdx.x;
  int plane = 2;
  while (plane > 0 && gu < fp->lr_unit_off[plane]) plane--;
  const int u = gu - fp->lr_unit_off[plane];
  Fit &F = fits[gu];
  if (threadIdx.x == 0) {
    unit_geom(fp, plane, u / fp->lr_unit_cols[plane], u % fp->lr_unit_cols[plane], &sh.geom);
    sh.cn = F.n;
  }
  for (int i = threadIdx.x; i < F.n * 6; i += THREADS) sh.ctaps[i / 6][i % 6] = F.taps[i / 6][i % 6];
  for (int i = threadIdx.x; i < F.n; i += THREADS) sh.csse[i] = F.sse[i];
  __syncthreads();
  const Geom g = sh.geom;
  const int n0 = sh.cn;
  int fitted[2][3], ref[2][3];
  for (int pass = 0; pass < 2; pass++)
    for (int j = 0; j < 3; j++) fitted[pass][j] = F.w[pass][j];
  bool staged = false;
  for (int q = 0; q < 3 && q <= u; q++) {
    for (int pass = 0; pass < 2; pass++)
      for (int j = 0; j < 3; j++) ref[pass][j] = q == 0 ? T(Wiener_Taps_Mid)[j] : fits[gu - q].w[pass][j];
    spec_path(fp, plane, g, cdef, dbk, src, fitted, ref, sh, staged);
  }
  __syncthreads();
  const int n1 = sh.cn;
  for (int i = n0 * 6 + threadIdx.x; i < n1 * 6; i += THREADS) F.taps[i / 6][i % 6] = sh.ctaps[i / 6][i % 6];
  for (int i = n0 + threadIdx.x; i < n1; i += THREADS) F.sse[i] = sh.csse[i];
  if (threadIdx.x == 0) F.n = n1;
}

__global__ void __launch_bounds__(THREADS) k_lr_select(FrameParams *fp, const uint8_t *cdef, const uint8_t *dbk,
                                                      const uint8_t *src, const Fit *fits, LrUnit *units,
                                                      int lrTest, int *lrTypes) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Shared &sh = *reinterpret_cast<Shared *>(smem_raw);
  const int plane = blockIdx.x;
  const int nUnits = fp->lr_unit_rows[plane] * fp->lr_unit_cols[plane], off = fp->lr_unit_off[plane];
  int refW[2][3], refX[2];
  for (int pass = 0; pass < 2; pass++) {
    refX[pass] = T(Sgrproj_Xqd_Mid)[pass];
    for (int j = 0; j < 3; j++) refW[pass][j] = T(Wiener_Taps_Mid)[j];
  }
  int used = 0;
  for (int u = 0; u < nUnits; u++) {
    __syncthreads();  // every thread is done with the previous unit's copy
    {  // the unit's first-pass results into shared memory (the rate scan reads them many times)
      const int *fs = reinterpret_cast<const int *>(fits + off + u);
      int *fd = reinterpret_cast<int *>(&sh.fit);
      for (int k = threadIdx.x; k < (int)(sizeof(Fit) / 4); k += THREADS) fd[k] = fs[k];
    }
    const Fit &F = sh.fit;
    Geom g;
    if (threadIdx.x == 0) unit_geom(fp, plane, u / fp->lr_unit_cols[plane], u % fp->lr_unit_cols[plane], &sh.geom);
    __syncthreads();
    g = sh.geom;
    __syncthreads();
    LrUnit best = {};
    best.type = RESTORE_NONE;
    long long bestCost = rd(fp, F.sse_none, 1);
    int tw[2][3], tx[2];
    LrUnit w = wiener_unit(F.w);
    bool staged = false;
    memcpy(tw, refW, sizeof tw);
    memcpy(tx, refX, sizeof tx);
    long long wc = rd(fp, F.sse[0], 2 + unit_bits(plane, w, tw, tx));
    for (int pass = 0; pass < 2; pass++)
      for (int j = plane ? 1 : 0; j < 3; j++)
        for (int d = -1; d <= 1; d += 2) {
          LrUnit t = w;
          t.wiener[pass][j] += d;
          if (t.wiener[pass][j] < T(Wiener_Taps_Min)[j] || t.wiener[pass][j] > T(Wiener_Taps_Max)[j]) continue;
          memcpy(tw, refW, sizeof tw);
          memcpy(tx, refX, sizeof tx);
          long long tc = rd(fp, wiener_sse(fp, F, g, cdef, dbk, src, t, sh, staged), 2 + unit_bits(plane, t, tw, tx));
          if (tc < wc) {
            wc = tc;
            w = t;
          }
        }
    if (wc < bestCost) {
      bestCost = wc;
      best = w;
    }
    for (int set = 0; set < 16; set++) {
      LrUnit s = {};
      s.type = RESTORE_SGRPROJ;
      s.set = set;
      s.xqd[0] = F.xqd[set][0];
      s.xqd[1] = F.xqd[set][1];
      memcpy(tw, refW, sizeof tw);
      memcpy(tx, refX, sizeof tx);
      long long sc = rd(fp, F.sgr_sse[set], 2 + unit_bits(plane, s, tw, tx));
      if (sc < bestCost) {
        bestCost = sc;
        best = s;
      }
    }
    if (lrTest) {
      // Wiener on even units, the self-guided set of least SSE on odd ones
      if (!(u & 1)) {
        best = w;
      } else {
        long long bs = -1;
        for (int set = 0; set < 16; set++) {
          long long v = F.sgr_sse[set];
          if (bs < 0 || v < bs) {
            bs = v;
            best = LrUnit{};
            best.type = RESTORE_SGRPROJ;
            best.set = set;
            best.xqd[0] = F.xqd[set][0];
            best.xqd[1] = F.xqd[set][1];
          }
        }
      }
    }
    unit_bits(plane, best, refW, refX);
    if (threadIdx.x == 0) units[off + u] = best;
    used |= best.type != RESTORE_NONE;
  }
  if (threadIdx.x == 0) fp->lr_type[plane] = lrTypes[plane] = used ? RESTORE_SWITCHABLE : RESTORE_NONE;
}

}  // namespace lrs
