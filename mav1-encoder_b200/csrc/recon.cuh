// Closed-loop reconstruction (reference src/kernels/k_recon.h,
// scheduled by src/backend_cpu.c:76-156).
//
// Per block in decode order: prediction (inter: 8-tap / compound average /
// optional 3x3 dual-filter search; intra: per transform block from the
// reconstructed neighbours with the spec's BlockDecoded availability),
// forward transform by the Q20 matrices, dead-zone quantisation, eob, and
// the normative inverse transform added back into `rec`; optional luma
// transform-type search and intra tx_depth search by 16 * SSE + lambda * bits.
//
// B200 mapping, two launches per frame:
//  - k_recon_inter: a 128-thread CTA per superblock codes its inter blocks
//    (they read reference pictures only, so every superblock starts at once)
//    and publishes each block's completion flags;
//  - k_recon_blocks: the intra blocks as dataflow. A prepass (k_block_map,
//    k_block_order, k_block_deps) maps every 4x4 unit to its block, lists the
//    intra blocks, and gives each one its dependency count (the intra blocks
//    under its luma edge samples, spec 7.11.2 aboveLimit / leftLimit), its
//    place in those blocks' successor lists and the BlockDecoded bits of its
//    corner units; blocks without dependencies seed a ready queue. Persistent
//    128-thread workers (at most one per SM, max(8, intra blocks / 8) of
//    them) pop ready blocks, stage each one in shared memory in one batch of
//    copies, code its luma, write it back, publish its luma flag and release
//    its successors (the last release pushes a successor to the queue), then
//    wait (bounded) on the chroma flags under its chroma edges and code its
//    chroma. Every wait is bounded (Ctx::spin_limit polls); past it the
//    worker sets the error and abort words and every worker stops.
// BlockDecoded availability is a function of the decode order (the unit map
// and the corner bits) or of the clear-flags rule (k_recon.h:402-414)
// outside the superblock. Samples of the frame being written are read
// through L2 (ldpx), as other SMs write them during the launch. Within a
// transform block the CTA splits the residual, both matrix passes (64-bit
// accumulation), the quantiser, the eob search (a max over inverse-scan
// positions), the row / column inverse kernels and the reconstruction.
#pragma once

#include "common.cuh"
#include "pred.cuh"
#include "tx.cuh"

namespace rec {

// Threads of the CTA coding a block: INTER_THREADS for the inter blocks of a
// superblock, INTRA_THREADS for an intra block worker.
#define RT ((int)blockDim.x)
#ifndef MAV1CU_INTER_THREADS
#define MAV1CU_INTER_THREADS 128
#endif
#ifndef MAV1CU_INTRA_THREADS
#define MAV1CU_INTRA_THREADS 128
#endif
constexpr int INTER_THREADS = MAV1CU_INTER_THREADS, INTRA_THREADS = MAV1CU_INTRA_THREADS;
#define FWD_SLOT_SIZE 4096
HD int fwd_slot(int kind, int log2n) { return (kind * 5 + log2n - 2) * FWD_SLOT_SIZE; }

// inverse scan tables: position -> scan index, per (scan class, tx size)
__constant__ int d_inv_scan_off[3][19];
__device__ int16_t d_inv_scan[8192];

HD int scan_class(int t) {
  if (t == V_DCT || t == V_ADST || t == V_FLIPADST) return 1;
  if (t == H_DCT || t == H_ADST || t == H_FLIPADST) return 2;
  return 0;
}

struct Ctx {
  const FrameParams *fp;
  const uint8_t *src;
  uint8_t *rec;
  const uint8_t *ref, *gold;
  BlockInfo *blocks;
  const SbInfo *sbs;
  int32_t *coefs;
  const int32_t *mats;
  const int32_t *mats_t;  // the same matrices transposed
  int *status;          // [0] error (1 ready-queue wait, 2 successor list, 3 chroma-edge wait, 4 bulk copy), [1] abort
  const int *blk_at;    // per 4x4 luma unit of the frame: index of the block covering it
  int *done;            // per block index: 1 once its luma samples are written; then the same for chroma
  // the intra blocks' ready queue: unfinished luma dependencies per block,
  // successor lists (blocks whose luma edges read this block's luma), and
  // the queue of blocks whose luma dependencies are all complete (slot
  // value: block index + 1; 0 while the slot is unfilled)
  int *dep_count, *succ_count, *succ;
  int *queue, *qtail;
  // per intra block, BlockDecoded of its corner units: bit 0 / 1 luma
  // above-right / below-left, bit 2 / 3 the same for chroma
  int *corners;
  // polls a dependency wait makes before it gives up (sets the error and
  // abort words); SPIN_LIMIT unless a test shortens it
  int spin_limit;
  // a block index whose luma dependencies are counted once more than they
  // are, so it is never released (-1: none): the failure-detection test's
  // never-released dependency
  int hold;
};

#define MAX_SUCC 96  // successors per block: at most 25 along each edge, with margin

#define TILE_OFF 4     // tile column of the block's first sample (word aligned; the left column at 3)
#define TILE_Y 132     // luma tile stride: TILE_OFF + 2 * 64; rows -1 .. 127
#define TILE_C 68      // chroma tile stride: TILE_OFF + 2 * 32; rows -1 .. 63
#define FMAT_SMALL 336 // 4 * 4 + 8 * 8 + 16 * 16

struct Smem {
  int32_t resid[64 * 64];  // residual, then the inverse transform's plane
  int32_t tmp[64 * 32];    // forward row pass output
  int32_t q[32 * 32];      // levels of the current candidate
  int32_t qbest[32 * 32];  // levels kept by the tx type search
  int sse33[33];
  long long red[(INTER_THREADS > INTRA_THREADS ? INTER_THREADS : INTRA_THREADS) / 32];  // one per warp
  BlockInfo blk;
  int maxLumaW, maxLumaH;
  int flag;
  int me;      // index of the block being coded
  int r0, c0;  // its superblock's first 4x4 row / column
  // views of the reconstruction and the source: plane origins (absolute
  // plane coordinates) and strides; the frames for an inter block, the
  // tiles below for an intra block
  uint8_t *recp[3];
  int rstride[3];
  const uint8_t *srcp[3];
  int sstride[3];
  FrameParams fpc;           // the CTA's copy of the frame parameters
  uint64_t qinv[3][2];       // per plane: the quantiser's reciprocals of dc_q and ac_q (tx::quant_inv)
  int cornerAR[3], cornerBL[3];  // BlockDecoded of those units
  // What only one of the two kernels uses. k_recon_inter launches with the
  // shared memory up to the end of its part (SMEM_INTER), k_recon_blocks
  // with the whole struct, so neither holds the other's part on its SMs.
  union {
    struct {  // inter blocks
      int16_t pred0[64 * 64];  // first compound prediction (intermediate precision)
      // the superblock's source (luma 64 x 64, then the two 32 x 32 chroma
      // planes), bulk-copied in once per CTA
      __align__(16) uint8_t srcSB[64 * 64 + 2 * 32 * 32];
      // the block plane being coded: prediction, then reconstruction, then
      // written back to the frame
      __align__(16) uint8_t recT[64 * 64];
      __align__(8) unsigned long long bar;  // completion of the source copies
    };
    struct {  // intra blocks
      int32_t fmat[3][FMAT_SMALL];   // forward matrices of lengths 4, 8, 16 per kind
      int32_t fmatT[3][FMAT_SMALL];  // the same transposed
      int cbits;               // the block's corner bits (Ctx::corners)
      int succN;               // its successor count and list, copied while staging
      int succ[MAX_SUCC];
      int edge[3][EDGE_LEN];   // AboveRow, LeftCol, filter copy
      uint8_t save[64 * 64];   // the block's luma before the tx_depth candidates
      // tiles: rows and columns -1 .. 2n - 1 around the block (its own
      // samples, the above row over the above-right units, the left column
      // over the below-left units), and its source
      uint8_t tileY[TILE_Y * 129];
      uint8_t tileC[2][TILE_C * 65];
      uint8_t srcY[64 * 64];
      uint8_t srcC[2][32 * 32];
    };
  };
};
constexpr size_t SMEM_INTER = offsetof(Smem, bar) + sizeof(unsigned long long);
constexpr size_t SMEM_INTRA = sizeof(Smem);

// Sums / maxima over the CTA. A one-warp CTA reduces by shuffles alone; the
// __syncwarp()s order the shared-memory writes before and after like the
// block barriers of the general path.
__device__ __forceinline__ long long cta_sum64(long long v, Smem &sm) {
  if (blockDim.x == 32) __syncwarp();
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  if (blockDim.x == 32) {
    __syncwarp();
    return v;
  }
  if ((threadIdx.x & 31) == 0) sm.red[threadIdx.x >> 5] = v;
  __syncthreads();
  long long s = 0;
  for (int k = 0; k < RT / 32; k++) s += sm.red[k];
  __syncthreads();
  return s;
}
__device__ __forceinline__ int cta_max(int v, Smem &sm) {
  if (blockDim.x == 32) __syncwarp();
  for (int off = 16; off > 0; off >>= 1) v = imax(v, __shfl_xor_sync(0xffffffffu, v, off));
  if (blockDim.x == 32) {
    __syncwarp();
    return v;
  }
  if ((threadIdx.x & 31) == 0) sm.red[threadIdx.x >> 5] = v;
  __syncthreads();
  int m = 0;
  for (int k = 0; k < RT / 32; k++) m = imax(m, (int)sm.red[k]);
  __syncthreads();
  return m;
}

struct CtaSync {
  __device__ void operator()() const { __syncthreads(); }
};

// One row of the inverse transform at a fixed width: dequantised levels ->
// row transform -> clamp, into sm.resid (stride 64).
template <int LW>
__device__ void inv_row(Smem &sm, const int32_t *q, int i, int th, int dcQ, int acQ, int denom, int rect, int rk,
                        int rowShift) {
  constexpr int W = 1 << LW, TW = W < 32 ? W : 32;
  int32_t t[W];
  int nz = 0;
#pragma unroll
  for (int j = 0; j < W; j++) {
    t[j] = (j < TW && i < th) ? tx::dequant_level(q[i * TW + j], (i == 0 && j == 0) ? dcQ : acQ, denom) : 0;
    nz |= t[j];
  }
  if (!nz) {
#pragma unroll
    for (int j = 0; j < W; j++) sm.resid[i * 64 + j] = 0;
    return;
  }
  if (rect) {
#pragma unroll
    for (int j = 0; j < W; j++) t[j] = (int32_t)round2l((int64_t)t[j] * 2896, 12);
  }
  tx::inverse_1d_n<LW>(t, rk, 16);
#pragma unroll
  for (int j = 0; j < W; j++) sm.resid[i * 64 + j] = clip3(-(1 << 15), (1 << 15) - 1, round2(t[j], rowShift));
}

// One column at a fixed height: column transform, then either added into the
// reconstruction (flipped for FLIPADST types) or stored back into sm.resid.
template <int LH>
__device__ void inv_col(Smem &sm, int j, int w, int ck, int fud, int flr, uint8_t *rec, int rs, int x, int y) {
  constexpr int H = 1 << LH;
  int32_t t[H];
#pragma unroll
  for (int i = 0; i < H; i++) t[i] = sm.resid[i * 64 + j];
  tx::inverse_1d_n<LH>(t, ck, 16);
  if (rec) {
    uint8_t *col = rec + y * rs + x + (flr ? (w - 1 - j) : j);
#pragma unroll
    for (int i = 0; i < H; i++) {
      uint8_t *o = col + (fud ? (H - 1 - i) : i) * rs;
      *o = (uint8_t)clip1((int)*o + round2(t[i], 4));
    }
  } else {
#pragma unroll
    for (int i = 0; i < H; i++) sm.resid[i * 64 + j] = round2(t[i], 4);
  }
}

// The 32- and 64-point DCT rows / columns by two threads each (adjacent
// lanes of one warp; half 0 runs the even half and the first join pairs,
// half 1 the odd half and the rest, tx::idct_odd), which halves the
// sequential butterfly chain of the largest transforms. Each thread loads
// its permuted inputs directly; the pre-join halves meet in sm.resid.
template <int LW>
__device__ void inv_row_split(Smem &sm, const int32_t *q, int i, int half, int th, int dcQ, int acQ, int denom,
                              int rect, int rowShift) {
  constexpr int W = 1 << LW, HW = W / 2, TW = W < 32 ? W : 32;
  unsigned pair = 3u << ((threadIdx.x & 31) & ~1u);
  int32_t t[HW];
  int nz = 0;
#pragma unroll
  for (int k = 0; k < HW; k++) {
    int j = tx::brev(LW, k + half * HW);
    t[k] = (j < TW && i < th) ? tx::dequant_level(q[i * TW + j], (i == 0 && j == 0) ? dcQ : acQ, denom) : 0;
    nz |= t[k];
  }
  nz |= __shfl_xor_sync(pair, nz, 1);
  int32_t *row = sm.resid + i * 64;
  if (!nz) {
#pragma unroll
    for (int k = 0; k < HW; k++) row[k + half * HW] = 0;
    return;
  }
  if (rect) {
#pragma unroll
    for (int k = 0; k < HW; k++) t[k] = (int32_t)round2l((int64_t)t[k] * 2896, 12);
  }
  if (half == 0) tx::idct<LW - 1, false>(t, 16);
  else tx::idct_odd<LW>(t, 16);
#pragma unroll
  for (int k = 0; k < HW; k++) row[k + half * HW] = t[k];
  __syncwarp(pair);
#pragma unroll
  for (int k = 0; k < HW / 2; k++) {
    int a = k + half * (HW / 2), b = W - 1 - a;
    int32_t va = row[a], vb = row[b];
    tx::idct_join_pair(&va, &vb, 16);
    row[a] = clip3(-(1 << 15), (1 << 15) - 1, round2(va, rowShift));
    row[b] = clip3(-(1 << 15), (1 << 15) - 1, round2(vb, rowShift));
  }
}

template <int LH>
__device__ void inv_col_split(Smem &sm, int j, int half, int w, int fud, int flr, uint8_t *rec, int rs, int x, int y) {
  constexpr int H = 1 << LH, HH = H / 2;
  unsigned pair = 3u << ((threadIdx.x & 31) & ~1u);
  int32_t t[HH];
#pragma unroll
  for (int k = 0; k < HH; k++) t[k] = sm.resid[tx::brev(LH, k + half * HH) * 64 + j];
  __syncwarp(pair);  // both halves read before the column is overwritten
  if (half == 0) tx::idct<LH - 1, false>(t, 16);
  else tx::idct_odd<LH>(t, 16);
#pragma unroll
  for (int k = 0; k < HH; k++) sm.resid[(k + half * HH) * 64 + j] = t[k];
  __syncwarp(pair);
  uint8_t *col = rec ? rec + y * rs + x + (flr ? (w - 1 - j) : j) : nullptr;
#pragma unroll
  for (int k = 0; k < HH / 2; k++) {
    int a = k + half * (HH / 2), b = H - 1 - a;
    int32_t va = sm.resid[a * 64 + j], vb = sm.resid[b * 64 + j];
    tx::idct_join_pair(&va, &vb, 16);
    if (rec) {
      uint8_t *oa = col + (fud ? (H - 1 - a) : a) * rs, *ob = col + (fud ? (H - 1 - b) : b) * rs;
      *oa = (uint8_t)clip1((int)*oa + round2(va, 4));
      *ob = (uint8_t)clip1((int)*ob + round2(vb, 4));
    } else {
      sm.resid[a * 64 + j] = round2(va, 4);
      sm.resid[b * 64 + j] = round2(vb, 4);
    }
  }
}

// Levels of a candidate -> reconstruction residual (spec 7.13.3 with the
// dequantisation of 7.12.3), into sm.resid (stride 64).
// With rec set, the column pass adds its output straight into the
// reconstruction (flipped for FLIPADST types) instead of storing it.
// MAXL: the largest log2 length the instantiation handles; the sizes up to
// 16 get their own inlined copy, so their register allocation does not
// carry the 32- and 64-point kernels.
template <int MAXL>
__device__ __forceinline__ void inverse_2d_upto(Smem &sm, const int32_t *q, int txSz, int txType, int dcQ, int acQ,
                                                uint8_t *rec, int rs, int x, int y) {
  int lw = T(Tx_Width_Log2)[txSz], lh = T(Tx_Height_Log2)[txSz];
  int w = 1 << lw, h = 1 << lh, th = imin(32, h);
  int rowShift = T(Transform_Row_Shift)[txSz], denom = tx::dq_denom(txSz);
  int rect = iabs(lw - lh) == 1;
  int rk = tx::row_kind(txType), ck = tx::col_kind(txType);
  if (MAXL >= 5 && lw >= 5 && rk == tx::KIND_DCT) {
    for (int p = threadIdx.x; p < 2 * h; p += RT) {
      if (lw == 5) inv_row_split<5>(sm, q, p >> 1, p & 1, th, dcQ, acQ, denom, rect, rowShift);
      else inv_row_split<6>(sm, q, p >> 1, p & 1, th, dcQ, acQ, denom, rect, rowShift);
    }
  } else for (int i = threadIdx.x; i < h; i += RT) {
    switch (lw) {
      case 2: inv_row<2>(sm, q, i, th, dcQ, acQ, denom, rect, rk, rowShift); break;
      case 3: inv_row<3>(sm, q, i, th, dcQ, acQ, denom, rect, rk, rowShift); break;
      case 4: inv_row<4>(sm, q, i, th, dcQ, acQ, denom, rect, rk, rowShift); break;
      case 5: if (MAXL >= 5) inv_row<5>(sm, q, i, th, dcQ, acQ, denom, rect, rk, rowShift); break;
      default: if (MAXL >= 6) inv_row<6>(sm, q, i, th, dcQ, acQ, denom, rect, rk, rowShift); break;
    }
  }
  __syncthreads();
  int fud = tx::flip_ud(txType), flr = tx::flip_lr(txType);
  if (MAXL >= 5 && lh >= 5 && ck == tx::KIND_DCT) {
    for (int p = threadIdx.x; p < 2 * w; p += RT) {
      if (lh == 5) inv_col_split<5>(sm, p >> 1, p & 1, w, fud, flr, rec, rs, x, y);
      else inv_col_split<6>(sm, p >> 1, p & 1, w, fud, flr, rec, rs, x, y);
    }
  } else for (int j = threadIdx.x; j < w; j += RT) {
    switch (lh) {
      case 2: inv_col<2>(sm, j, w, ck, fud, flr, rec, rs, x, y); break;
      case 3: inv_col<3>(sm, j, w, ck, fud, flr, rec, rs, x, y); break;
      case 4: inv_col<4>(sm, j, w, ck, fud, flr, rec, rs, x, y); break;
      case 5: if (MAXL >= 5) inv_col<5>(sm, j, w, ck, fud, flr, rec, rs, x, y); break;
      default: if (MAXL >= 6) inv_col<6>(sm, j, w, ck, fud, flr, rec, rs, x, y); break;
    }
  }
  __syncthreads();
}

__device__ __noinline__ void inverse_2d_large(Smem &sm, const int32_t *q, int txSz, int txType, int dcQ, int acQ,
                                              uint8_t *rec, int rs, int x, int y) {
  inverse_2d_upto<6>(sm, q, txSz, txType, dcQ, acQ, rec, rs, x, y);
}

// A size up to 16 x 16 with both lengths (and the rectangular scaling)
// known at compile time: the passes of inverse_2d_upto for that size
// (dequantisation denominator 1), straight-line.
template <int LW, int LH>
__device__ __forceinline__ void inverse_2d_fixed(Smem &sm, const int32_t *q, int txType, int dcQ, int acQ,
                                                 int rowShift, uint8_t *rec, int rs, int x, int y) {
  constexpr int W = 1 << LW, H = 1 << LH, rect = LW - LH == 1 || LH - LW == 1;
  int rk = tx::row_kind(txType), ck = tx::col_kind(txType);
  for (int i = threadIdx.x; i < H; i += RT) inv_row<LW>(sm, q, i, H, dcQ, acQ, 1, rect, rk, rowShift);
  __syncthreads();
  int fud = tx::flip_ud(txType), flr = tx::flip_lr(txType);
  for (int j = threadIdx.x; j < W; j += RT) inv_col<LH>(sm, j, W, ck, fud, flr, rec, rs, x, y);
  __syncthreads();
}

// SMALL_INLINE: sizes up to 16 inlined, one fixed-size copy per size (the
// intra workers, whose chains wait on these latencies: a fixed-size 8x8
// inverse takes about 40% fewer cycles than the length-generic one);
// otherwise every size through the out-of-line copy (the inter kernel, where
// that keeps its register budget).
template <bool SMALL_INLINE>
__device__ __forceinline__ void inverse_2d(Smem &sm, const int32_t *q, int txSz, int txType, int dcQ, int acQ,
                                           uint8_t *rec = nullptr, int rs = 0, int x = 0, int y = 0) {
  if (threadIdx.x == 0) {  // h rows of w points, then w columns of h points: 3 log2 N operations per point
    int lw = T(Tx_Width_Log2)[txSz], lh = T(Tx_Height_Log2)[txSz];
    WORK(W_REC_INV_OPS, 3 * (1 << (lw + lh)) * (lw + lh));
  }
  if (SMALL_INLINE) {
    int rsh = T(Transform_Row_Shift)[txSz];
    switch (txSz) {
      case TX_4X4: inverse_2d_fixed<2, 2>(sm, q, txType, dcQ, acQ, rsh, rec, rs, x, y); return;
      case TX_8X8: inverse_2d_fixed<3, 3>(sm, q, txType, dcQ, acQ, rsh, rec, rs, x, y); return;
      case TX_16X16: inverse_2d_fixed<4, 4>(sm, q, txType, dcQ, acQ, rsh, rec, rs, x, y); return;
      case TX_4X8: inverse_2d_fixed<2, 3>(sm, q, txType, dcQ, acQ, rsh, rec, rs, x, y); return;
      case TX_8X4: inverse_2d_fixed<3, 2>(sm, q, txType, dcQ, acQ, rsh, rec, rs, x, y); return;
      case TX_8X16: inverse_2d_fixed<3, 4>(sm, q, txType, dcQ, acQ, rsh, rec, rs, x, y); return;
      case TX_16X8: inverse_2d_fixed<4, 3>(sm, q, txType, dcQ, acQ, rsh, rec, rs, x, y); return;
      case TX_4X16: inverse_2d_fixed<2, 4>(sm, q, txType, dcQ, acQ, rsh, rec, rs, x, y); return;
      case TX_16X4: inverse_2d_fixed<4, 2>(sm, q, txType, dcQ, acQ, rsh, rec, rs, x, y); return;
      default: break;
    }
  }
  inverse_2d_large(sm, q, txSz, txType, dcQ, acQ, rec, rs, x, y);
}

// Forward matrix of a kind and length: for the intra workers lengths 4..16
// from the CTA's shared copy, otherwise (and for the inter kernel, whose
// shared memory holds the superblock's source instead) from the table in
// global memory; fwd_matrix_t gives the transpose (the row pass reads it
// along the output index, so the lanes of a warp read consecutive words).
template <bool INTER>
__device__ __forceinline__ const int32_t *fwd_matrix(const Ctx &c, const Smem &sm, int kind, int lg) {
  return !INTER && lg <= 4 ? sm.fmat[kind] + (lg == 2 ? 0 : lg == 3 ? 16 : 80) : c.mats + fwd_slot(kind, lg);
}
template <bool INTER>
__device__ __forceinline__ const int32_t *fwd_matrix_t(const Ctx &c, const Smem &sm, int kind, int lg) {
  return !INTER && lg <= 4 ? sm.fmatT[kind] + (lg == 2 ? 0 : lg == 3 ? 16 : 80) : c.mats_t + fwd_slot(kind, lg);
}

// The transpose of every forward matrix (slot k: kind k / 5, length 4 << k % 5).
__global__ void k_transpose_mats(const int32_t *mats, int32_t *matsT) {
  int slot = blockIdx.x, n = 4 << (slot % 5);
  const int32_t *m = mats + slot * FWD_SLOT_SIZE;
  int32_t *t = matsT + slot * FWD_SLOT_SIZE;
  for (int e = threadIdx.x; e < n * n; e += blockDim.x) t[(e % n) * n + e / n] = m[e];
}

// Forward row pass at a fixed width: row i of the residual (sm.resid,
// stride 64) times the kept TW rows of the Q20 matrix (read from its
// transpose MhT), 64-bit sums rounded by 16 bits into sm.tmp (stride 32).
template <int LW>
__device__ void fwd_rows(Smem &sm, const int32_t *MhT, int h) {
  constexpr int W = 1 << LW, LTW = LW < 5 ? LW : 5, TW = 1 << LTW;
  for (int k = threadIdx.x; k < h * TW; k += RT) {
    int i = k >> LTW, kk = k & (TW - 1);
    const int32_t *r = sm.resid + i * 64, *m = MhT + kk;
    int64_t s = 0;
#pragma unroll
    for (int j = 0; j < W; j++) s += (int64_t)r[j] * m[j * W];
    sm.tmp[i * 32 + kk] = (int32_t)round2l(s, 16);
  }
}

// Forward column sum at a fixed height for output (k2, kk).
template <int LH>
__device__ __forceinline__ int64_t fwd_col(const Smem &sm, const int32_t *Mv, int k2, int kk) {
  constexpr int H = 1 << LH;
  const int32_t *m = Mv + k2 * H;
  int64_t s = 0;
#pragma unroll
  for (int i = 0; i < H; i++) s += (int64_t)m[i] * sm.tmp[i * 32 + kk];
  return s;
}

// Transform, quantise and reconstruct one transform block whose prediction
// is in `rec` (code_tx_block, k_recon.h:60-173). Returns the eob.
template <bool INTER>
__device__ __forceinline__ int code_tx(const Ctx &c, Smem &sm, const uint8_t *src, int stride, uint8_t *rec, int rs, int x, int y, int txSz,
                       int plane, const int *cands, int numCands, int32_t *coefOut, int *outType, long long *outCost) {
  const FrameParams *fp = c.fp;
  int lw = T(Tx_Width_Log2)[txSz], lh = T(Tx_Height_Log2)[txSz];
  int w = 1 << lw, h = 1 << lh, tw = imin(32, w), th = imin(32, h);
  int dcQ = fp->dc_q[plane], acQ = fp->ac_q[plane];
  int tid = threadIdx.x;
  if (fp->lossless) {
    // 4x4 Walsh-Hadamard, exact inverse of the spec's (k_fwd.h:112-136); one thread
    if (tid == 0) {
      int r[16], t[16];
      for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) r[i * 4 + j] = (int)src[(y + i) * stride + x + j] - (int)rec[(y + i) * rs + x + j];
      for (int j = 0; j < 4; j++) {
        int a1 = r[0 * 4 + j], b1 = r[1 * 4 + j], c1 = r[2 * 4 + j], d1 = r[3 * 4 + j];
        a1 += b1;
        d1 = d1 - c1;
        int e1 = (a1 - d1) >> 1;
        b1 = e1 - b1;
        c1 = e1 - c1;
        a1 -= c1;
        d1 += b1;
        t[0 * 4 + j] = a1; t[1 * 4 + j] = c1; t[2 * 4 + j] = d1; t[3 * 4 + j] = b1;
      }
      for (int i = 0; i < 4; i++) {
        int a1 = t[i * 4 + 0], b1 = t[i * 4 + 1], c1 = t[i * 4 + 2], d1 = t[i * 4 + 3];
        a1 += b1;
        d1 -= c1;
        int e1 = (a1 - d1) >> 1;
        b1 = e1 - b1;
        c1 = e1 - c1;
        a1 -= c1;
        d1 += b1;
        sm.q[i * 4 + 0] = a1; sm.q[i * 4 + 1] = c1; sm.q[i * 4 + 2] = d1; sm.q[i * 4 + 3] = b1;
      }
      int eob = 0;
      const int16_t *inv = d_inv_scan + d_inv_scan_off[0][TX_4X4];
      for (int k = 0; k < 16; k++) {
        coefOut[k] = sm.q[k];
        if (sm.q[k] != 0) eob = imax(eob, inv[k] + 1);
      }
      if (eob > 0) {
        int32_t rr[4][4];
        for (int i = 0; i < 4; i++) {
          int32_t tt[4];
          for (int j = 0; j < 4; j++) tt[j] = tx::dequant_level(sm.q[i * 4 + j], (i == 0 && j == 0) ? dcQ : acQ, 1);
          tx::iwht(tt, 2);
          for (int j = 0; j < 4; j++) rr[i][j] = tt[j];
        }
        for (int j = 0; j < 4; j++) {
          int32_t tt[4];
          for (int i = 0; i < 4; i++) tt[i] = clip3(-(1 << 15), (1 << 15) - 1, rr[i][j]);
          tx::iwht(tt, 0);
          for (int i = 0; i < 4; i++) rr[i][j] = tt[i];
        }
        for (int i = 0; i < 4; i++)
          for (int j = 0; j < 4; j++) {
            int o = (y + i) * rs + x + j;
            rec[o] = (uint8_t)clip1((int)rec[o] + rr[i][j]);
          }
      }
      sm.flag = eob;
    }
    __syncthreads();
    int eob = sm.flag;
    __syncthreads();
    *outType = DCT_DCT;
    *outCost = 0;
    return eob;
  }

  int single = numCands == 1 && !fp->tx_mode_select;
  int shifts = T(Transform_Row_Shift)[txSz] + 4, rect = iabs(lw - lh) == 1;
  int denom = tx::dq_denom(txSz);
  uint64_t invDc = sm.qinv[plane][0], invAc = sm.qinv[plane][1];  // derived once per CTA (load_shared)
  long long bestCost = -1;
  int bestType = DCT_DCT, bestEob = 0;
  int32_t *qsrc = sm.q;  // levels the final reconstruction uses
  for (int ci = 0; ci < numCands; ci++) {
    int t = cands[ci];
    int fud = tx::flip_ud(t), flr = tx::flip_lr(t);
    for (int k = tid; k < h * w; k += RT) {
      int i = k >> lw, j = k & (w - 1);
      int yy = fud ? (h - 1 - i) : i, xx = flr ? (w - 1 - j) : j;
      sm.resid[i * 64 + j] = (int)src[(y + yy) * stride + x + xx] - (int)rec[(y + yy) * rs + x + xx];
    }
    __syncthreads();
    const int32_t *Mh = fwd_matrix_t<INTER>(c, sm, tx::row_kind(t), lw), *Mv = fwd_matrix<INTER>(c, sm, tx::col_kind(t), lh);
    if (tid == 0) {  // row pass h x tw outputs of w terms, column pass th x tw outputs of h terms
      WORK(W_REC_FWD_MAC, h * tw * w + th * tw * h);
      WORK(W_REC_QUANT, th * tw);
    }
    switch (lw) {
      case 2: fwd_rows<2>(sm, Mh, h); break;
      case 3: fwd_rows<3>(sm, Mh, h); break;
      case 4: fwd_rows<4>(sm, Mh, h); break;
      case 5: fwd_rows<5>(sm, Mh, h); break;
      default: fwd_rows<6>(sm, Mh, h); break;
    }
    __syncthreads();
    const int16_t *inv = d_inv_scan + d_inv_scan_off[scan_class(t)][txSz];
    int myEob = 0, myNz = 0;
    int ltw = imin(5, lw);
    for (int k = tid; k < th * tw; k += RT) {
      int k2 = k >> ltw, kk = k & (tw - 1);
      int64_t s;
      switch (lh) {
        case 2: s = fwd_col<2>(sm, Mv, k2, kk); break;
        case 3: s = fwd_col<3>(sm, Mv, k2, kk); break;
        case 4: s = fwd_col<4>(sm, Mv, k2, kk); break;
        case 5: s = fwd_col<5>(sm, Mv, k2, kk); break;
        default: s = fwd_col<6>(sm, Mv, k2, kk); break;
      }
      s = s * ((int64_t)1 << shifts);
      if (rect) s = round2l(s, 12) * 5793;
      int v = (int)(s >= 0 ? round2l(s, 20) : -round2l(-s, 20));
      int first = k == 0;
      int lv = tx::quant_level(v, first ? dcQ : acQ, first ? 26 : 22, denom, first ? invDc : invAc);
      sm.q[k] = lv;
      myNz |= lv != 0;
      if (!single && lv != 0) myEob = imax(myEob, inv[k] + 1);
    }
    if (single) {
      // only "has coefficients" matters here (the writer derives the eob)
      int nz = __syncthreads_or(myNz);
      for (int k = tid; k < tw * th; k += RT) coefOut[k] = sm.q[k];
      if (nz) inverse_2d<!INTER>(sm, sm.q, txSz, t, dcQ, acQ, rec, rs, x, y);
      *outType = nz ? t : DCT_DCT;
      *outCost = 0;
      return nz;
    }
    int eob = cta_max(myEob, sm);  // includes the barrier after the quantiser
    long long sse = 0;
    if (eob > 0) {
      // keep the residual-free path's SSE source intact: the inverse reuses resid
      inverse_2d<!INTER>(sm, sm.q, txSz, t, dcQ, acQ);
      for (int k = tid; k < h * w; k += RT) {
        int i = k >> lw, j = k & (w - 1);
        int yy = fud ? (h - 1 - i) : i, xx = flr ? (w - 1 - j) : j;
        int d = (int)src[(y + yy) * stride + x + xx] - clip1((int)rec[(y + yy) * rs + x + xx] + sm.resid[i * 64 + j]);
        sse += d * d;
      }
    } else {
      for (int k = tid; k < h * w; k += RT) {
        int i = k >> lw, j = k & (w - 1);
        int d = sm.resid[i * 64 + j];
        sse += d * d;
      }
    }
    sse = cta_sum64(sse, sm);
    long long bits = 0;
    if (eob == 0) {
      bits = tid == 0 ? 8 : 0;
    } else {
      for (int k = tid; k < th * tw; k += RT)
        if (inv[k] < eob) {
          int l = iabs(sm.q[k]);
          bits += l == 0 ? 6 : 8 * (2 + 2 * floor_log2(l));
        }
      if (tid == 0) bits += 8 * 6 + 8 * 2 * floor_log2(eob + 1);
    }
    bits = cta_sum64(bits, sm);
    long long cost = sse * 16 + (long long)fp->lambda * bits / 8;
    if (bestCost < 0 || cost < bestCost) {
      bestCost = cost;
      bestType = eob > 0 ? t : DCT_DCT;
      bestEob = eob;
      for (int k = tid; k < tw * th; k += RT) sm.qbest[k] = sm.q[k];
      qsrc = sm.qbest;
      __syncthreads();
    }
  }
  for (int k = tid; k < tw * th; k += RT) coefOut[k] = qsrc[k];
  if (bestEob > 0) {
    int fud = tx::flip_ud(bestType), flr = tx::flip_lr(bestType);
    if (numCands > 1) inverse_2d<!INTER>(sm, qsrc, txSz, bestType, dcQ, acQ);
    for (int k = tid; k < h * w; k += RT) {
      int i = k >> lw, j = k & (w - 1);
      int yy = fud ? (h - 1 - i) : i, xx = flr ? (w - 1 - j) : j;
      int o = (y + yy) * rs + x + xx;
      rec[o] = (uint8_t)clip1((int)rec[o] + sm.resid[i * 64 + j]);
    }
  }
  __syncthreads();
  *outType = bestType;
  *outCost = bestCost;
  return bestEob;
}

__device__ __forceinline__ void tx_type_set(BlockInfo &b, int idx, int t) {
  if (idx >= 16) return;
  int sh = 4 * (idx & 7);
  if (idx < 8) b.tx_types_lo = (int32_t)(((uint32_t)b.tx_types_lo & ~(15u << sh)) | ((uint32_t)t << sh));
  else b.tx_types_hi = (int32_t)(((uint32_t)b.tx_types_hi & ~(15u << sh)) | ((uint32_t)t << sh));
}

// CfL alpha of one chroma transform block: first minimum of the SSE over
// alpha in [-16, 16] (cfl_best_alpha, k_intra.h:277-313).
__device__ int cfl_alpha(Smem &sm, const uint8_t *luma, int ls, int startX, int startY, int maxLumaW, int maxLumaH,
                         int log2W, int log2H, int dcv, const uint8_t *sp, int stride, int excludeZero, int *avgOut) {
  int w = 1 << log2W, h = 1 << log2H, n = w * h;
  long long sum = 0;
  for (int k = threadIdx.x; k < n; k += RT) sum += pred::cfl_luma(luma, ls, startX, startY, maxLumaW, maxLumaH, k >> log2W, k & (w - 1));
  int avg = round2((int)cta_sum64(sum, sm), log2W + log2H);
  int sse[33];
  for (int a = 0; a < 33; a++) sse[a] = 0;
  for (int k = threadIdx.x; k < n; k += RT) {
    int i = k >> log2W, j = k & (w - 1);
    int v = pred::cfl_luma(luma, ls, startX, startY, maxLumaW, maxLumaH, i, j) - avg;
    int s0 = sp[i * stride + j];
    for (int a = 0; a < 33; a++) {
      int d = clip3(0, 255, dcv + round2signed((a - 16) * v, 6)) - s0;
      sse[a] += d * d;
    }
  }
  for (int a = threadIdx.x; a < 33; a += RT) sm.sse33[a] = 0;
  __syncthreads();
  for (int a = 0; a < 33; a++) {
    int v = sse[a];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(&sm.sse33[a], v);
  }
  __syncthreads();
  long long best = -1;
  int bestA = 0;
  for (int a = -16; a <= 16; a++) {
    if (a == 0 && excludeZero) continue;
    long long s = sm.sse33[a + 16];
    if (best < 0 || s < best) {
      best = s;
      bestA = a;
    }
  }
  __syncthreads();
  *avgOut = avg;
  return bestA;
}

// The clear-flags value of a unit outside the superblock (superblock-relative
// units of the plane, -1..n): clear_block_decoded_flags (k_recon.h:402-414).
__device__ __forceinline__ int decoded_outside(const FrameParams *fp, int r0, int c0, int sub, int y, int x) {
  int n = 16 >> sub;
  if (y == n && x == -1) return 0;
  if (y < 0) return x < ((tile_col_end(fp, c0) - c0) >> sub);
  if (x < 0) return y < ((fp->mi_rows - r0) >> sub);
  return 0;
}

// BlockDecoded of the above-right (k = 0) or below-left (k = 1) corner unit of
// plane p of block b (index me, superblock origin r0, c0) from the frame's
// unit map: the clear-flags value outside the superblock, else whether the
// block covering it precedes this one.
__device__ __forceinline__ int corner_decoded(const FrameParams *fp, const int *blkAt, const BlockInfo &b, int me,
                                              int r0, int c0, int p, int k) {
  int sub = p > 0, n = 16 >> sub;
  int top = (b.mi_row & 15) >> sub, left = (b.mi_col & 15) >> sub;
  int y = k ? top + (block_h(b.bsize) >> (2 + sub)) : top - 1;
  int x = k ? left - 1 : left + (block_w(b.bsize) >> (2 + sub));
  if (y < 0 || x < 0 || y >= n || x >= n) return decoded_outside(fp, r0, c0, sub, y, x);
  int r = r0 + (y << sub), col = c0 + (x << sub);
  if (r >= fp->mi_rows || col >= fp->mi_cols) return 0;
  int blk = blkAt[r * fp->mi_cols + col];
  return blk >= 0 && blk < me;
}

// The edge samples plane p of block b can read (see stage_chroma_edges): row ay
// from ax0 to ax1 and column x0 - 1 from ly0 to ly1 (empty runs: end <
// start), and the 4x4 luma units under them as two runs (ur, uc, urow, un).
struct EdgeRuns {
  int ay, ax0, ax1, ly0, ly1;
  int ur[2], uc[2], urow[2], un[2];
};
__device__ __forceinline__ EdgeRuns edge_runs(const FrameParams *fp, const BlockInfo &b, int p, int ar, int bl) {
  EdgeRuns e;
  int bs = b.bsize, sub = p > 0, w = block_w(bs) >> sub, h = block_h(bs) >> sub;
  int availU = b.mi_row > 0, availL = b.mi_col > tile_col_start(fp, b.mi_col);
  int x0 = (b.mi_col >> sub) * 4, y0 = (b.mi_row >> sub) * 4;
  int txSz = fp->lossless ? TX_4X4 : sub ? uv_tx_size(bs, 1, 1) : T(Max_Tx_Size_Rect)[bs];
  int ext = imin(T(Tx_Width)[txSz], T(Tx_Height)[txSz]);
  int maxX = ((fp->mi_cols * 4) >> sub) - 1, maxY = ((fp->mi_rows * 4) >> sub) - 1;
  e.ay = y0 - 1;
  e.ax0 = x0 - availL;
  e.ax1 = availU ? imin(maxX, x0 + w - 1 + (ar ? ext : 0)) : e.ax0 - 1;
  e.ly0 = y0 - availU;
  e.ly1 = availL ? imin(maxY, y0 + h - 1 + (bl ? ext : 0)) : e.ly0 - 1;
  e.ur[0] = (e.ay << sub) >> 2;
  e.uc[0] = (e.ax0 << sub) >> 2;
  e.urow[0] = 1;
  e.un[0] = e.ax1 >= e.ax0 ? ((e.ax1 << sub) >> 2) - e.uc[0] + 1 : 0;
  e.ur[1] = (e.ly0 << sub) >> 2;
  e.uc[1] = ((x0 - 1) << sub) >> 2;
  e.urow[1] = 0;
  e.un[1] = e.ly1 >= e.ly0 ? ((e.ly1 << sub) >> 2) - e.ur[1] + 1 : 0;
  return e;
}

// BlockDecoded[plane][y][x] (superblock-relative units of the plane, -1..n)
// as the reference's flags hold it when block sm.blk codes a transform
// block. Outside the superblock: the clear-flags values. Inside, a unit is
// decoded when the block covering it precedes this one in decode order. The
// queries (above-right / below-left of a transform block) land on this
// block itself, directly above it or left of it (blocks there precede it),
// directly right of it or below it (they follow it), or on the block's
// above-right / below-left corner unit, looked up once per block in
// stage_begin. `own` answers for a unit of this block: its transform blocks
// run in raster order, so the unit above-right of one is coded (1) and the
// unit below-left is not (0). Units beyond the frame report 0: the edge
// limits clip to maxX / maxY there, so their flag is never used.
__device__ int decoded(const Ctx &c, const Smem &sm, int plane, int y, int x, int own) {
  const FrameParams *fp = c.fp;
  int sub = plane > 0, n = 16 >> sub;
  if (y < 0 || x < 0 || y >= n || x >= n) return decoded_outside(fp, sm.r0, sm.c0, sub, y, x);
  if (sm.r0 + (y << sub) >= fp->mi_rows || sm.c0 + (x << sub) >= fp->mi_cols) return 0;
  const BlockInfo &b = sm.blk;
  int top = (b.mi_row & 15) >> sub, left = (b.mi_col & 15) >> sub;
  int bottom = top + (block_h(b.bsize) >> (2 + sub)), right = left + (block_w(b.bsize) >> (2 + sub));
  if (y >= top && y < bottom && x >= left && x < right) return own;
  if (y == top - 1 && x == right) return sm.cornerAR[plane];
  if (y == bottom && x == left - 1) return sm.cornerBL[plane];
  return y < top || x < left;
}

#define SPIN_LIMIT (1 << 22)  // polls of at least one L2 round trip each: about a second (Ctx::spin_limit)

// Block index covering 4x4 luma unit (r, col) (the frame's map, built
// before the launch).
__device__ __forceinline__ int block_at(const Ctx &c, const Smem &, int r, int col) {
  return __ldg(c.blk_at + r * c.fp->mi_cols + col);
}

// Waits until the block covering each 4x4 unit of up to 6 runs of units
// has completed the planes of `group` (0: luma, 1: chroma)
// (run k: first (r[k], col[k]), along a row if row[k], else a column;
// n[k] units), unless it is this block. Lanes take units of
// all runs at once. Every block waited on precedes this one in the claim
// order (or is an inter block, complete before the launch), so the wait
// ends; past the limit it sets the error and abort words and gives up,
// and every other wait then stops too.
__device__ void wait_units(const Ctx &c, const Smem &sm, int group, const int *r, const int *col, const int *row,
                           const int *n) {
  int nblk = c.fp->sb_cols * c.fp->sb_rows * MAX_BLOCKS_PER_SB;
  volatile const int *vdone = c.done + group * nblk;
  volatile int *vstatus = c.status;
  int total = n[0] + n[1] + n[2] + n[3] + n[4] + n[5];
  for (int i = threadIdx.x; i < total; i += RT) {
    int k = 0, j = i;
    while (j >= n[k]) j -= n[k++];
    int b = block_at(c, sm, r[k] + (row[k] ? 0 : j), col[k] + (row[k] ? j : 0));
    if (b == sm.me || (unsigned)b >= (unsigned)nblk) continue;
    int spins = 0;
    while (!vdone[b]) {
      if (vstatus[1] || ++spins > c.spin_limit) {
        if (!vstatus[1]) {
          atomicExch(c.status, 3);  // 3: a chroma-edge wait gave up
          atomicExch(c.status + 1, 1);
        }
        break;
      }
      __nanosleep(64);
    }
  }
}

// A run of 32-bit words to copy from global to shared memory: n words,
// 2^lgw per row, row strides gs (global) / ds (shared) bytes.
struct CopySeg {
  uint8_t *dst;
  const uint8_t *src;
  int ds, gs, n, lgw;
};

// Copies up to NS runs at once through L2 (__ldcg: the frame is being
// written by other SMs): each lane issues the loads of a batch of words
// from any of the runs before its stores, so the whole copy costs about one
// L2 round trip per batch.
#define COPY_BATCH 8
template <int NS>
__device__ void copy_segs(const CopySeg *sg) {
  int total = 0;
#pragma unroll
  for (int k = 0; k < NS; k++) total += sg[k].n;
  for (int base = 0; base < total; base += RT * COPY_BATCH) {
    uint32_t v[COPY_BATCH];
    uint32_t *d[COPY_BATCH];
#pragma unroll
    for (int m = 0; m < COPY_BATCH; m++) {
      int j = base + m * RT + (int)threadIdx.x, k = 0;
      d[m] = nullptr;
      if (j >= total) continue;
#pragma unroll
      for (int q = 0; q < NS - 1; q++)
        if (k == q && j >= sg[q].n) {
          j -= sg[q].n;
          k = q + 1;
        }
      const CopySeg &g = sg[k];
      int r = j >> g.lgw, w = j & ((1 << g.lgw) - 1);
      v[m] = __ldcg((const unsigned *)(g.src + r * g.gs + 4 * w));
      d[m] = (uint32_t *)(g.dst + r * g.ds + 4 * w);
    }
#pragma unroll
    for (int m = 0; m < COPY_BATCH; m++)
      if (d[m]) *d[m] = v[m];
  }
}

// The copies of plane p's edge samples (edge runs e, see stage_chroma_edges)
// into its tile: the row above from the word holding its first sample, and
// the column left as the word ending at it, one per row.
__device__ __forceinline__ void edge_segs(const Ctx &c, Smem &sm, int p, const EdgeRuns &e, CopySeg *sg) {
  const FrameParams *fp = c.fp;
  const BlockInfo &b = sm.blk;
  int sub = p > 0, S = sub ? TILE_C : TILE_Y;
  uint8_t *t = sub ? sm.tileC[p - 1] : sm.tileY;
  int x0 = (b.mi_col >> sub) * 4, y0 = (b.mi_row >> sub) * 4, fs = fp->stride[p];
  const uint8_t *g = c.rec + fp->offset[p];
  int xs = e.ax0 & ~3;
  sg[0] = CopySeg{t + xs - x0 + TILE_OFF, g + e.ay * fs + xs, 0, 0, e.ax1 >= e.ax0 ? ((e.ax1 - xs) >> 2) + 1 : 0, 20};
  sg[1] = CopySeg{t + (e.ly0 - y0 + 1) * S + TILE_OFF - 4, g + e.ly0 * fs + x0 - 4, S, fs,
                  e.ly1 >= e.ly0 ? e.ly1 - e.ly0 + 1 : 0, 0};
}

// Stages an intra block in shared memory, in one batch of copies: the
// block's own samples of every plane (the reconstruction so far, overwritten
// as it is coded), its source, its luma edge samples and its successor list.
// The luma edges are complete: the ready queue hands out a block only once
// every block under them has published its luma (k_block_deps). The corner
// units' BlockDecoded come from the prepass (sm.cbits); the views then point
// at the tiles.
__device__ void stage_begin(const Ctx &c, Smem &sm) {
  const FrameParams *fp = c.fp;
  const BlockInfo &b = sm.blk;
  int bs = b.bsize, tid = threadIdx.x, cb = sm.cbits;
  CopySeg sg[10];
  int ns = 0;
  for (int p = 0; p < 3; p++) {
    int sub = p > 0, S = sub ? TILE_C : TILE_Y;
    uint8_t *t = sub ? sm.tileC[p - 1] : sm.tileY, *sb = sub ? sm.srcC[p - 1] : sm.srcY;
    int lw = floor_log2(block_w(bs) >> sub), w = 1 << lw, h = block_h(bs) >> sub;
    int x0 = (b.mi_col >> sub) * 4, y0 = (b.mi_row >> sub) * 4, fs = fp->stride[p];
    sg[ns++] = CopySeg{t + S + TILE_OFF, c.rec + fp->offset[p] + y0 * fs + x0, S, fs, (w >> 2) * h, lw - 2};
    sg[ns++] = CopySeg{sb, c.src + fp->offset[p] + y0 * fs + x0, w, fs, (w >> 2) * h, lw - 2};
    if (tid == 0) {
      sm.recp[p] = t + S + TILE_OFF - ((ptrdiff_t)y0 * S + x0);
      sm.rstride[p] = S;
      sm.srcp[p] = sb - ((ptrdiff_t)y0 * w + x0);
      sm.sstride[p] = w;
    }
  }
  if (tid < 3) {
    int sh = tid ? 2 : 0;
    sm.cornerAR[tid] = (cb >> sh) & 1;
    sm.cornerBL[tid] = (cb >> (sh + 1)) & 1;
  }
  edge_segs(c, sm, 0, edge_runs(fp, b, 0, cb & 1, (cb >> 1) & 1), sg + ns);
  ns += 2;
  sg[ns++] = CopySeg{(uint8_t *)sm.succ, (const uint8_t *)(c.succ + (size_t)sm.me * MAX_SUCC), 0, 0, MAX_SUCC, 20};
  sg[ns++] = CopySeg{(uint8_t *)&sm.succN, (const uint8_t *)(c.succ_count + sm.me), 0, 0, 1, 0};
  copy_segs<10>(sg);
  __syncthreads();
}

// The chroma planes' edge samples, once the blocks that wrote them have
// completed their chroma. Those are the row above and the column left of the
// block, extended past its corner by the largest candidate transform's
// shorter side where the above-right / below-left unit is decoded: the union
// of the samples intra_edges reads (above / left limits, spec 7.11.2) over
// every transform block of every candidate size. Copies move whole aligned
// words (a word of the row above or of the column left may carry samples no
// transform block reads). The luma edges are staged with the block.
__device__ void stage_chroma_edges(const Ctx &c, Smem &sm) {
  const FrameParams *fp = c.fp;
  const BlockInfo &b = sm.blk;
  EdgeRuns e[2];
  int ur[6] = {0}, uc[6] = {0}, urow[6] = {0}, un[6] = {0};  // the 4x4 luma units under the edge samples
  for (int q = 0; q < 2; q++) {
    e[q] = edge_runs(fp, b, 1 + q, sm.cornerAR[1 + q], sm.cornerBL[1 + q]);
    for (int k = 0; k < 2; k++) {
      ur[2 * q + k] = e[q].ur[k];
      uc[2 * q + k] = e[q].uc[k];
      urow[2 * q + k] = e[q].urow[k];
      un[2 * q + k] = e[q].un[k];
    }
  }
  wait_units(c, sm, 1, ur, uc, urow, un);
  __threadfence();
  __syncthreads();
  CopySeg sg[4];
  edge_segs(c, sm, 1, e[0], sg);
  edge_segs(c, sm, 2, e[1], sg + 2);
  copy_segs<4>(sg);
  __syncthreads();
}

// Writes planes p0 .. p1 - 1 of an intra block's own samples from its tiles
// to the frame (whole words: block positions and widths are multiples of 4
// samples), then publishes them complete (flag group 0: luma, 1: chroma).
__device__ void unstage_intra(const Ctx &c, Smem &sm, int p0, int p1) {
  const FrameParams *fp = c.fp;
  const BlockInfo &b = sm.blk;
  for (int p = p0; p < p1; p++) {
    int sub = p > 0, S = sub ? TILE_C : TILE_Y;
    const uint8_t *t = sub ? sm.tileC[p - 1] : sm.tileY;
    int lw = floor_log2(block_w(b.bsize) >> sub) - 2, h = block_h(b.bsize) >> sub;
    int x0 = (b.mi_col >> sub) * 4, y0 = (b.mi_row >> sub) * 4, fs = fp->stride[p];
    uint8_t *g = c.rec + fp->offset[p] + y0 * fs + x0;
    for (int k = threadIdx.x; k < (h << lw); k += RT) {
      int i = k >> lw, j = k & ((1 << lw) - 1);
      *(uint32_t *)(g + i * fs + 4 * j) = *(const uint32_t *)(t + (i + 1) * S + TILE_OFF + 4 * j);
    }
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) atomicExch(c.done + (p0 ? fp->sb_cols * fp->sb_rows * MAX_BLOCKS_PER_SB : 0) + sm.me, 1);
}

// Every transform block of one plane of block b (code_plane, k_recon.h:190-291).
template <bool INTER>
__device__ long long code_plane(const Ctx &c, Smem &sm, int plane, int txSz) {
  const FrameParams *fp = c.fp;
  BlockInfo &b = sm.blk;
  int bs = b.bsize, MiRow = b.mi_row, MiCol = b.mi_col;
  int AvailU = MiRow > 0, AvailL = MiCol > tile_col_start(fp, MiCol);
  int sub = plane > 0;
  int planeSz = T(Subsampled_Size)[bs][sub][sub];
  int num4x4W = T(Num_4x4_Blocks_Wide)[planeSz], num4x4H = T(Num_4x4_Blocks_High)[planeSz];
  int baseX = (MiCol >> sub) * 4, baseY = (MiRow >> sub) * 4;
  int stride = sm.sstride[plane];           // source view
  const uint8_t *spx = sm.srcp[plane];
  uint8_t *px = sm.recp[plane];             // reconstruction view
  int rs = sm.rstride[plane];
  int stepX = T(Tx_Width)[txSz] >> 2, stepY = T(Tx_Height)[txSz] >> 2;
  int cands[16], numCands = 0;
  const int isInter = INTER;
  if (plane == 0) {
    int set = get_tx_set(txSz, isInter, fp->reduced_tx_set);
    if (!fp->tx_search || set == TX_SET_DCTONLY || fp->lossless) {
      cands[numCands++] = DCT_DCT;
    } else {
      for (int t = 0; t < 16; t++)
        if (tx_type_in_set(set, t, isInter)) cands[numCands++] = t;
    }
  } else {
    cands[numCands++] = chroma_tx_type(txSz, isInter, b.uv_mode, b.tx_type, fp->reduced_tx_set);
  }
  long long total = 0;
  int txIdx = 0, anyNz = 0;
  int *above = sm.edge[0] + EDGE_OFF, *left = sm.edge[1] + EDGE_OFF, *etmp = sm.edge[2];
  for (int y = 0; y < num4x4H; y += stepY) {
    for (int x = 0; x < num4x4W; x += stepX) {
      int startX = baseX + 4 * x, startY = baseY + 4 * y;
      if (startX >= ((fp->mi_cols * 4) >> sub) || startY >= ((fp->mi_rows * 4) >> sub)) continue;
      int row = (startY << sub) >> 2, col = (startX << sub) >> 2;
      int sbr = row & 15, sbc = col & 15;
      if (!isInter) {
        pred::IntraArgs a;
        a.haveLeft = AvailL || x > 0;
        a.haveAbove = AvailU || y > 0;
        a.haveAboveRight = decoded(c, sm, plane, (sbr >> sub) - 1, (sbc >> sub) + stepX, 1);
        a.haveBelowLeft = decoded(c, sm, plane, (sbr >> sub) + stepY, (sbc >> sub) - 1, 0);
        int isCfl = plane > 0 && b.uv_mode == UV_CFL_PRED;
        a.mode = plane == 0 ? b.y_mode : (isCfl ? DC_PRED : b.uv_mode);
        a.angleDelta = plane == 0 ? b.angle_y : b.angle_uv;
        a.log2W = T(Tx_Width_Log2)[txSz];
        a.log2H = T(Tx_Height_Log2)[txSz];
        a.maxX = ((fp->mi_cols * 4) >> sub) - 1;
        a.maxY = ((fp->mi_rows * 4) >> sub) - 1;
        a.edgeFilter = fp->enable_intra_edge_filter;
        a.filterType = (b.interp_filter >> (plane == 0 ? 4 : 5)) & 1;
        pred::IntraState st;
        pred::intra_state(a, &st);
        pred::intra_edges(px, rs, startX, startY, a, st, above, left, etmp, (int)threadIdx.x, RT, CtaSync());
        int tw = 1 << a.log2W, th = 1 << a.log2H;
        int dcv = a.mode == DC_PRED ? pred::intra_dc(a, above, left) : 0;
        uint8_t *d = px + startY * rs + startX;
        if (threadIdx.x == 0) WORK(W_REC_INTRA_PX, tw * th);
        for (int k = threadIdx.x; k < tw * th; k += RT) {
          int i = k >> a.log2W, j = k & (tw - 1);
          d[i * rs + j] = (uint8_t)(a.mode == DC_PRED ? dcv : pred::intra_pixel(a, st, above, left, i, j));
        }
        __syncthreads();
        if (isCfl) {
          const uint8_t *luma = sm.recp[0];
          int ls = sm.rstride[0];
          int alpha, avg;
          if (txIdx > 0) {
            alpha = plane == 1 ? b.cfl_alpha_u : b.cfl_alpha_v;
            int n = tw * th;
            long long sum = 0;
            for (int k = threadIdx.x; k < n; k += RT)
              sum += pred::cfl_luma(luma, ls, startX, startY, sm.maxLumaW, sm.maxLumaH, k >> a.log2W, k & (tw - 1));
            avg = round2((int)cta_sum64(sum, sm), a.log2W + a.log2H);
          } else {
            alpha = cfl_alpha(sm, luma, ls, startX, startY, sm.maxLumaW, sm.maxLumaH, a.log2W, a.log2H, dcv,
                              spx + startY * stride + startX, stride, plane == 2 && b.cfl_alpha_u == 0, &avg);
            if (threadIdx.x == 0) {
              if (plane == 1) b.cfl_alpha_u = alpha;
              else b.cfl_alpha_v = alpha;
            }
          }
          for (int k = threadIdx.x; k < tw * th; k += RT) {
            int i = k >> a.log2W, j = k & (tw - 1);
            int v = pred::cfl_luma(luma, ls, startX, startY, sm.maxLumaW, sm.maxLumaH, i, j);
            d[i * rs + j] = (uint8_t)pred::cfl_pixel(dcv, alpha, v, avg);
          }
          __syncthreads();
        }
      }
      if (plane == 0 && threadIdx.x == 0) {
        sm.maxLumaW = startX + stepX * 4;
        sm.maxLumaH = startY + stepY * 4;
      }
      int t = DCT_DCT;
      long long cst = 0;
      int eob = code_tx<INTER>(c, sm, spx, stride, px, rs, startX, startY, txSz, plane, cands, numCands,
                        c.coefs + b.coef_off[plane] + txIdx * T(Tx_Width)[txSz] * T(Tx_Height)[txSz], &t, &cst);
      total += cst;
      if (threadIdx.x == 0 && plane == 0) {
        tx_type_set(b, txIdx, t);
        if (txIdx == 0) b.tx_type = t;
      }
      txIdx++;
      anyNz |= eob > 0;
      __syncthreads();
    }
  }
  if (threadIdx.x == 0) b.eob[plane] = anyNz;
  __syncthreads();
  return total;
}

// Inter prediction of a w x h block (spec 7.11.3.4), staged: the clamped
// reference window (h + 7 rows of w + 7 samples) in shared memory, the
// horizontal 8-tap pass of every window row (Round2 by InterRound0 = 3), then
// the vertical pass per output sample - the values inter_sum forms sample
// by sample (k_inter.h:451-504). mode 0: final samples (Round2 by 11,
// clipped) into d (stride ds); 1: compound intermediates (Round2 by 7) into
// sm.pred0; 2: Round2(pred0 + this block's intermediates, 5), clipped, into
// d. Scratch: sm.tmp (window), sm.resid (horizontal pass).
__device__ void predict_block(Smem &sm, const pred::Inter &ip, int lw, int h, int mode, uint8_t *d, int ds) {
  int w = 1 << lw, W = w + 7, H = h + 7;
  uint8_t *win = (uint8_t *)sm.tmp;
  if (threadIdx.x == 0) WORK(W_REC_INTER_PX, w * h);
  int16_t *hs = (int16_t *)sm.resid;
  for (int k = threadIdx.x; k < W * H; k += RT) {
    int R = k / W, C = k - R * W;
    win[k] = ip.ref[(size_t)clip3(0, ip.lastY, ip.iy0 + R) * ip.stride + clip3(0, ip.lastX, ip.ix0 + C)];
  }
  __syncthreads();
  for (int k = threadIdx.x; k < H * w; k += RT) {
    int R = k >> lw, cc = k & (w - 1);
    const uint8_t *row = win + R * W + cc;
    int s = 0;
#pragma unroll
    for (int t = 0; t < 8; t++) s += ip.fh[t] * (int)row[t];
    hs[k] = (int16_t)round2(s, 3);
  }
  __syncthreads();
  for (int k = threadIdx.x; k < h * w; k += RT) {
    int r = k >> lw, cc = k & (w - 1);
    int acc = 0;
#pragma unroll
    for (int tv = 0; tv < 8; tv++) acc += ip.fv[tv] * (int)hs[(r + tv) * w + cc];
    if (mode == 0) d[r * ds + cc] = (uint8_t)clip1(round2(acc, 11));
    else if (mode == 1) sm.pred0[k] = (int16_t)round2(acc, 7);
    else d[r * ds + cc] = (uint8_t)clip1(round2((int)sm.pred0[k] + round2(acc, 7), 5));
  }
  __syncthreads();
}


// ---- bulk copies (the TMA engine's cp.async.bulk) into shared memory ------------------
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

// One row copy global -> shared, completing on the mbarrier: both addresses
// 16-byte aligned, bytes a multiple of 16 (checked by the caller's layout).
__device__ __forceinline__ void bulk_row(void *dst, const void *src, unsigned bytes, unsigned long long *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Waits (bounded) for phase `parity` of the mbarrier to complete; false if
// it did not within `limit` polls.
__device__ __forceinline__ bool bar_wait(unsigned long long *bar, unsigned parity, int limit) {
  for (int i = 0; i < limit; i++) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// The superblock's source (luma 64 rows of 64 bytes, two chroma planes of
// 32 rows of 32 bytes) into sm.srcSB: one bulk copy per row, a thread each,
// all completing on sm.bar. Rows are 16-byte aligned in the padded frame
// layout (luma stride sb_cols * 64, chroma sb_cols * 32, superblock columns
// at multiples of 64 / 32 bytes, plane offsets multiples of 64). On a wait
// past the limit the error and abort words are set (status 4) and the copies
// are waited for again before the CTA goes on, so none lands after it.
__device__ void stage_sb_source(const Ctx &c, Smem &sm, int sb) {
  static_assert(INTER_THREADS == 128, "one thread per source row");
  const FrameParams *fp = c.fp;
  int sbr = sb / fp->sb_cols, sbc = sb % fp->sb_cols, t = threadIdx.x;
  if (t == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&sm.bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(&sm.bar)),
                 "r"(64 * 64 + 2 * 32 * 32)
                 : "memory");
  }
  __syncthreads();
  if (t < 64) {
    bulk_row(sm.srcSB + t * 64, c.src + fp->offset[0] + (size_t)(sbr * 64 + t) * fp->stride[0] + sbc * 64, 64, &sm.bar);
  } else {
    int p = 1 + ((t - 64) >> 5), r = (t - 64) & 31;
    bulk_row(sm.srcSB + 64 * 64 + (p - 1) * 32 * 32 + r * 32,
             c.src + fp->offset[p] + (size_t)(sbr * 32 + r) * fp->stride[p] + sbc * 32, 32, &sm.bar);
  }
  if (!bar_wait(&sm.bar, 0, c.spin_limit)) {
    if (t == 0) {
      atomicExch(c.status, 4);
      atomicExch(c.status + 1, 1);
    }
    bar_wait(&sm.bar, 0, c.spin_limit);
  }
}

// The inter block's plane p: views of the staged source (absolute plane
// coordinates into sm.srcSB) and of sm.recT (the block's own w x h samples).
__device__ __forceinline__ void inter_views(const Ctx &c, Smem &sm, int p) {
  const BlockInfo &b = sm.blk;
  int sub = p > 0, S = sub ? 32 : 64;
  int sbx = (sm.c0 * 4) >> sub, sby = (sm.r0 * 4) >> sub;
  const uint8_t *tile = sm.srcSB + (sub ? 64 * 64 + (p - 1) * 32 * 32 : 0);
  int w = block_w(b.bsize) >> sub, x0 = (b.mi_col >> sub) * 4, y0 = (b.mi_row >> sub) * 4;
  sm.srcp[p] = tile - ((ptrdiff_t)sby * S + sbx);
  sm.sstride[p] = S;
  sm.recp[p] = sm.recT - ((ptrdiff_t)y0 * w + x0);
  sm.rstride[p] = w;
}

// Writes plane p of the inter block back from sm.recT to the frame (whole
// words: block positions and widths are multiples of 4 samples).
__device__ void unstage_inter(const Ctx &c, Smem &sm, int p) {
  const FrameParams *fp = c.fp;
  const BlockInfo &b = sm.blk;
  int sub = p > 0, lw = floor_log2(block_w(b.bsize) >> sub) - 2, h = block_h(b.bsize) >> sub;
  int x0 = (b.mi_col >> sub) * 4, y0 = (b.mi_row >> sub) * 4, fs = fp->stride[p];
  uint8_t *g = c.rec + fp->offset[p] + y0 * fs + x0;
  for (int k = threadIdx.x; k < (h << lw); k += RT) {
    int i = k >> lw, j = k & ((1 << lw) - 1);
    *(uint32_t *)(g + i * fs + 4 * j) = *(const uint32_t *)(sm.recT + (i << (lw + 2)) + 4 * j);
  }
  __syncthreads();
}

// Appends a block whose luma dependencies are complete to the ready queue.
__device__ __forceinline__ void push_ready(const Ctx &c, int blk) {
  int t = atomicAdd(c.qtail, 1);
  __threadfence();  // the luma this release follows is visible before the slot fills
  atomicExch(c.queue + t, blk + 1);
}

// After this block's luma is published: one dependency fewer for each
// successor; the last one releases it to the ready queue.
__device__ void release_successors(const Ctx &c, const Smem &sm) {
  int n = imin(sm.succN, MAX_SUCC);  // the list staged with the block
  for (int k = threadIdx.x; k < n; k += RT) {
    int s = sm.succ[k];
    if (atomicSub(c.dep_count + s, 1) == 1) push_ready(c, s);
  }
}

// One block (recon_block, k_recon.h:293-394); sm.blk holds it.
template <bool INTER>
__device__ void recon_block(const Ctx &c, Smem &sm, BlockInfo *gb) {
  const FrameParams *fp = c.fp;
  BlockInfo &b = sm.blk;
  int bs = b.bsize;
  int comp = INTER && b.ref_frame1 > INTRA_FRAME;
  const uint8_t *ref = (INTER && b.ref_frame != LAST_FRAME) ? c.gold : c.ref;
  const uint8_t *ref1 = c.gold;
  int MiRow = b.mi_row, MiCol = b.mi_col;
  if (threadIdx.x == 0) {
    sm.maxLumaW = sm.maxLumaH = 0;
    b.tx_depth = 0;
    b.interp_filter &= 0x30;
  }
  // inter blocks: the superblock's staged source and the block tile
  // (one plane at a time, written back after it is coded)
  if (INTER && threadIdx.x < 3) inter_views(c, sm, threadIdx.x);
  __syncthreads();
  if (!INTER) stage_begin(c, sm);
  int tid = threadIdx.x;
  if (INTER && fp->switchable_interp && !comp) {
    int w = block_w(bs), h = block_h(bs);
    int x0 = MiCol * 4, y0 = MiRow * 4, stride = fp->stride[0], ss = sm.sstride[0], rs = sm.rstride[0];
    uint8_t *px = sm.recp[0] + y0 * rs + x0;
    const uint8_t *sp = sm.srcp[0] + y0 * ss + x0;
    int vw = imin(w, fp->frame_w - x0), vh = imin(h, fp->frame_h - y0);
    long long best = -1;
    int bestPacked = 0;
    for (int f = 0; f < 9; f++) {
      int packed = (f % 3) | ((f / 3) << 2);
      pred::Inter ip;
      pred::inter_setup(&ip, ref + fp->offset[0], stride, fp->frame_w, fp->frame_h, x0, y0, w, h, b.mv_row, b.mv_col,
                        0, 0, packed);
      long long sse = 0;
      predict_block(sm, ip, floor_log2(w), h, 0, px, rs);
      for (int k = tid; k < w * h; k += RT) {
        int i = k / w, j = k % w;
        if (i < vh && j < vw) {
          int d = (int)px[i * rs + j] - (int)sp[i * ss + j];
          sse += d * d;
        }
      }
      sse = cta_sum64(sse, sm);
      long long cst = sse * 16 + (long long)fp->lambda * ((f % 3 != 0) + (f / 3 != 0));
      if (best < 0 || cst < best) {
        best = cst;
        bestPacked = packed;
      }
    }
    if (tid == 0) b.interp_filter = bestPacked;
    __syncthreads();
  }
  for (int plane = 0; plane < 3; plane++) {
    if (plane == 1 && !INTER) {
      // luma is final: publish it, so blocks waiting only on it go ahead
      // while this one codes its chroma
      unstage_intra(c, sm, 0, 1);
      release_successors(c, sm);
      stage_chroma_edges(c, sm);
    }
    int sub = plane > 0, stride = fp->stride[plane];
    int baseX = (MiCol >> sub) * 4, baseY = (MiRow >> sub) * 4;
    if (INTER) {
      int w = block_w(bs) >> sub, h = block_h(bs) >> sub;
      int rs = sm.rstride[plane];
      uint8_t *d = sm.recp[plane] + baseY * rs + baseX;
      pred::Inter p0, p1;
      pred::inter_setup(&p0, ref + fp->offset[plane], stride, fp->frame_w, fp->frame_h, baseX, baseY, w, h, b.mv_row,
                        b.mv_col, sub, sub, b.interp_filter);
      if (comp)
        pred::inter_setup(&p1, ref1 + fp->offset[plane], stride, fp->frame_w, fp->frame_h, baseX, baseY, w, h,
                          b.mv1_row, b.mv1_col, sub, sub, b.interp_filter);
      if (comp) {
        predict_block(sm, p0, floor_log2(w), h, 1, d, rs);
        predict_block(sm, p1, floor_log2(w), h, 2, d, rs);
      } else {
        predict_block(sm, p0, floor_log2(w), h, 0, d, rs);
      }
    }
    int maxDepth = (!INTER && fp->tx_mode_select && !fp->lossless && plane == 0)
                       ? imin(MAX_TX_DEPTH, T(Max_Tx_Depth)[bs])
                       : 0;
    if (maxDepth == 0) {
      code_plane<INTER>(c, sm, plane,
                        fp->lossless ? TX_4X4 : plane > 0 ? uv_tx_size(bs, 1, 1) : T(Max_Tx_Size_Rect)[bs]);
      if (INTER) unstage_inter(c, sm, plane);
      continue;
    }
    // tx_depth RD search: every depth from the same pixels (BlockDecoded
    // inside the block follows the depth's own transform order), the winner
    // re-coded last unless it already was
    int w = block_w(bs), h = block_h(bs);
    int rs = sm.rstride[0];
    uint8_t *px = sm.recp[0] + baseY * rs + baseX;
    for (int k = tid; k < w * h; k += RT) sm.save[k] = px[(k / w) * rs + (k % w)];
    __syncthreads();
    long long best = -1;
    int bestD = 0;
    for (int d = 0; d <= maxDepth + 1; d++) {
      int depth = d <= maxDepth ? d : bestD;
      if (d == maxDepth + 1 && bestD == maxDepth) break;
      if (d > 0) {
        for (int k = tid; k < w * h; k += RT) px[(k / w) * rs + (k % w)] = sm.save[k];
        __syncthreads();
      }
      long long cst = code_plane<INTER>(c, sm, 0, depth_tx_size(bs, depth)) + (long long)fp->lambda * 8 * depth;
      if (d <= maxDepth && (best < 0 || cst < best)) {
        best = cst;
        bestD = depth;
      }
      if (d == maxDepth + 1) break;
    }
    if (tid == 0) b.tx_depth = bestD;
    __syncthreads();
  }
  if (!INTER) unstage_intra(c, sm, 1, 3);
  if (tid == 0) *gb = b;
}

// Per frame, before the recon launch: the block index of every 4x4 luma
// unit of the frame (one warp per superblock, lanes over a block's units).
__global__ void k_block_map(const FrameParams *fp, const BlockInfo *blocks, const SbInfo *sbs, int *blkAt) {
  int sb = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (sb >= fp->sb_cols * fp->sb_rows) return;
  SbInfo sbi = sbs[sb];
  int cols = fp->mi_cols, rows = fp->mi_rows;
  for (int k = 0; k < imin(sbi.num_blocks, MAX_BLOCKS_PER_SB); k++) {
    int idx = sb * MAX_BLOCKS_PER_SB + k;
    const BlockInfo &b = blocks[idx];
    if (b.mi_row < 0 || b.mi_col < 0) continue;
    int h = imax(0, imin(T(Num_4x4_Blocks_High)[b.bsize], rows - b.mi_row));
    int w = imax(0, imin(T(Num_4x4_Blocks_Wide)[b.bsize], cols - b.mi_col));
    for (int i = lane; i < w * h; i += 32) blkAt[(b.mi_row + i / w) * cols + b.mi_col + i % w] = idx;
  }
}

// The claim list of the intra workers: the frame's intra blocks,
// superblocks in wave order and decode order inside each (a prefix sum of
// the superblocks' intra block counts over one CTA), and its length.
__device__ __forceinline__ int intra_count(const BlockInfo *blocks, const SbInfo *sbs, int sb) {
  int n = imax(0, imin(sbs[sb].num_blocks, MAX_BLOCKS_PER_SB)), m = 0;
  for (int k = 0; k < n; k++) m += !blocks[sb * MAX_BLOCKS_PER_SB + k].is_inter;
  return m;
}
__global__ void __launch_bounds__(1024) k_block_order(const BlockInfo *blocks, const SbInfo *sbs, const int *order,
                                                      int nsb, int *list, int *total) {
  __shared__ int part[1024];
  int t = threadIdx.x, per = (nsb + 1023) / 1024, s0 = imin(nsb, t * per), s1 = imin(nsb, s0 + per);
  int sum = 0;
  for (int i = s0; i < s1; i++) sum += intra_count(blocks, sbs, order[i]);
  part[t] = sum;
  __syncthreads();
  for (int off = 1; off < 1024; off <<= 1) {
    int v = t >= off ? part[t - off] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int base = part[t] - sum;
  for (int i = s0; i < s1; i++) {
    int sb = order[i], n = imax(0, imin(sbs[sb].num_blocks, MAX_BLOCKS_PER_SB));
    for (int k = 0; k < n; k++)
      if (!blocks[sb * MAX_BLOCKS_PER_SB + k].is_inter) list[base++] = sb * MAX_BLOCKS_PER_SB + k;
  }
  if (t == 1023) *total = part[1023];
}

// The CTA's shared copies of the frame parameters, the quantiser's
// reciprocals and (intra workers) the forward matrices of lengths 4..16;
// returns the context reading them.
template <bool INTER>
__device__ Ctx load_shared(const Ctx &c, Smem &sm) {
  const int *src = (const int *)c.fp;
  int *dst = (int *)&sm.fpc;
  for (int k = threadIdx.x; k < (int)(sizeof(FrameParams) / 4); k += RT) dst[k] = src[k];
  Ctx cs = c;
  cs.fp = &sm.fpc;
  // the reciprocals are 64-bit divisions: once per CTA, not per transform block
  if (threadIdx.x < 6) {
    int p = threadIdx.x >> 1, q = (threadIdx.x & 1) ? c.fp->ac_q[p] : c.fp->dc_q[p];
    sm.qinv[p][threadIdx.x & 1] = q > 0 ? tx::quant_inv(q) : 0;
  }
  if (!INTER)  // the inter kernel's shared memory ends before the intra part
    for (int kind = 0; kind < 3; kind++)
      for (int lg = 2; lg <= 4; lg++) {
        int n = 1 << (2 * lg), off = lg == 2 ? 0 : lg == 3 ? 16 : 80;
        for (int k = threadIdx.x; k < n; k += RT) {
          sm.fmat[kind][off + k] = c.mats[fwd_slot(kind, lg) + k];
          sm.fmatT[kind][off + k] = c.mats_t[fwd_slot(kind, lg) + k];
        }
      }
  __syncthreads();
  return cs;
}



// The inter blocks of the frame, one CTA per superblock (all at once: they
// read reference pictures only), each published complete for the intra
// workers that read its samples.
__global__ void __launch_bounds__(INTER_THREADS, 512 / INTER_THREADS) k_recon_inter(Ctx cg) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem &sm = *(Smem *)smem_raw;
  const Ctx c = load_shared<true>(cg, sm);
  int sb = blockIdx.x, n = imax(0, imin(c.sbs[sb].num_blocks, MAX_BLOCKS_PER_SB));
  if (threadIdx.x == 0) {
    sm.r0 = (sb / c.fp->sb_cols) * 16;
    sm.c0 = (sb % c.fp->sb_cols) * 16;
  }
  stage_sb_source(c, sm, sb);
  for (int k = 0; k < n; k++) {
    int me = sb * MAX_BLOCKS_PER_SB + k;
    if (threadIdx.x == 0) sm.blk = c.blocks[me];
    __syncthreads();
    if (sm.blk.is_inter) {
      recon_block<true>(c, sm, c.blocks + me);
      __threadfence();
      __syncthreads();
      if (threadIdx.x == 0) {
        atomicExch(c.done + me, 1);
        atomicExch(c.done + c.fp->sb_cols * c.fp->sb_rows * MAX_BLOCKS_PER_SB + me, 1);
      }
    }
    __syncthreads();
  }
}

// Per frame, after the claim list: each intra block's dependencies (one
// warp per block). The blocks under its luma and chroma edge samples
// (edge_runs with its corner units' BlockDecoded) that are intra and not
// itself, without repeats: their number is its dependency count, and it
// joins each one's successor list. A block is released once all of them
// have published their luma; by then each of them is held by a worker, so
// the chroma waits that follow always end. Blocks with none start in the
// ready queue.
__global__ void __launch_bounds__(128) k_block_deps(Ctx c, const int *list, const int *total) {
  __shared__ int cand[4][160];
  const FrameParams *fp = c.fp;
  int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int item = blockIdx.x * 4 + warp; item < *total; item += gridDim.x * 4) {
    int me = list[item];
    BlockInfo b = c.blocks[me];
    int sb = me / MAX_BLOCKS_PER_SB, r0 = (sb / fp->sb_cols) * 16, c0 = (sb % fp->sb_cols) * 16;
    EdgeRuns e[2];  // luma; chroma (both chroma planes share their geometry)
    int cb = 0;
    for (int p = 0; p < 2; p++) {
      int ar = corner_decoded(fp, c.blk_at, b, me, r0, c0, p, 0), bl = corner_decoded(fp, c.blk_at, b, me, r0, c0, p, 1);
      e[p] = edge_runs(fp, b, p, ar, bl);
      cb |= (ar | bl << 1) << (2 * p);
    }
    if (lane == 0) c.corners[me] = cb;
    int run[4] = {e[0].un[0], e[0].un[1], e[1].un[0], e[1].un[1]};
    int n = imin(160, run[0] + run[1] + run[2] + run[3]);
    int nblk = fp->sb_cols * fp->sb_rows * MAX_BLOCKS_PER_SB;
    for (int i = lane; i < n; i += 32) {
      int k = 0, j = i;
      while (j >= run[k]) j -= run[k++];
      const EdgeRuns &er = e[k >> 1];
      int kk = k & 1;
      int r = er.ur[kk] + (er.urow[kk] ? 0 : j), col = er.uc[kk] + (er.urow[kk] ? j : 0);
      int d = c.blk_at[r * fp->mi_cols + col];
      if (d == me || (unsigned)d >= (unsigned)nblk || c.blocks[d].is_inter) d = -1;
      cand[warp][i] = d;
    }
    __syncwarp();
    int cnt = 0;
    for (int i = lane; i < n; i += 32) {
      int d = cand[warp][i];
      if (d < 0) continue;
      bool dup = false;
      for (int j = 0; j < i && !dup; j++) dup = cand[warp][j] == d;
      if (dup) continue;
      cnt++;
      int slot = atomicAdd(c.succ_count + d, 1);
      if (slot < MAX_SUCC) {
        c.succ[d * MAX_SUCC + slot] = me;
      } else {
        atomicExch(c.status, 2);
        atomicExch(c.status + 1, 1);
      }
    }
    for (int off = 16; off > 0; off >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, off);
    cnt += me == c.hold;
    if (lane == 0) {
      if (cnt == 0) push_ready(c, me);
      else c.dep_count[me] = cnt;
    }
    __syncwarp();
  }
}

// Claim state of the recon launch: the list, its length and the counter.
#ifndef MAV1CU_BLOCKS_PER_WORKER
#define MAV1CU_BLOCKS_PER_WORKER 8
#endif
#ifndef MAV1CU_MIN_WORKERS
#define MAV1CU_MIN_WORKERS 8
#endif
constexpr int BLOCKS_PER_WORKER = MAV1CU_BLOCKS_PER_WORKER, MIN_WORKERS = MAV1CU_MIN_WORKERS;

struct Claim {
  const int *list;
  const int *total;
  int *next;
};

// Every intra block of the frame, one persistent launch: each worker CTA
// takes the next slot of the ready queue, waits (bounded) until a released
// block fills it, stages and codes that block (its luma, published with its
// successors released, then its chroma) and publishes its completion flags.
__global__ void __launch_bounds__(INTRA_THREADS, 1) k_recon_blocks(Ctx cg, Claim q) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // workers in proportion to the frame's intra blocks: the surplus CTAs
  // leave at once, so their SMs' registers and shared memory go to the other
  // engines' kernels (an ALTREF frame has a few hundred intra blocks, a key
  // frame tens of thousands)
  int total = *q.total;
  if (blockIdx.x >= imax(MIN_WORKERS, total / BLOCKS_PER_WORKER)) return;
  Smem &sm = *(Smem *)smem_raw;
  const Ctx c = load_shared<false>(cg, sm);
  const FrameParams *fp = c.fp;
  volatile int *vstatus = c.status;
  for (;;) {
    if (threadIdx.x == 0) {
      int slot = vstatus[1] ? total : atomicAdd(q.next, 1), me = -1;
      if (slot < total) {
        // the slot fills once its block is released (every block is, once
        // the blocks before it in any dependency chain complete)
        // the value that ended the wait is the block: no second read of the
        // slot after the fence (one L2 round trip less per block)
        volatile int *vslot = c.queue + slot;
        int spins = 0, v;
        while (!(v = *vslot) && !vstatus[1]) {
          if (++spins > c.spin_limit) {
            atomicExch(c.status, 1);
            atomicExch(c.status + 1, 1);
            break;
          }
          __nanosleep(64);
        }
        __threadfence();
        me = v - 1;
      }
      sm.flag = me;
      if (me >= 0) {
        int sb = me / MAX_BLOCKS_PER_SB;
        sm.me = me;
        sm.r0 = (sb / fp->sb_cols) * 16;
        sm.c0 = (sb % fp->sb_cols) * 16;
        sm.blk = c.blocks[me];
        sm.cbits = c.corners[me];
      }
    }
    __syncthreads();
    int me = sm.flag;
    if (me < 0) return;
    recon_block<false>(c, sm, c.blocks + me);  // publishes its luma, then its chroma
    __syncthreads();
  }
}

}  // namespace rec
