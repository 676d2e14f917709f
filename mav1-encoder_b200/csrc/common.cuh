// Shared definitions of the mav1cu kernels: AV1 enumerations, the normative
// constant tables (device copies in constant / global memory, host copies for
// the host helpers) and the integer helpers every stage uses. All arithmetic
// is integer and mirrors the AV1 specification's definitions (Round2, Clip3,
// FloorLog2, ...), the same operations the reference encoder's kernels use
// (src/kernels/k_common.h:37-46).
#pragma once

#include <stdint.h>

#include "mav1cu.h"
#include "spec_tables_gen.h"

#if defined(__CUDACC__)
#define HD __host__ __device__ __forceinline__
#define HDM __host__ __device__ __forceinline__
#else
#define HD static inline
#define HDM inline
#endif

typedef mav1cu_frame_params FrameParams;
typedef mav1cu_block_info BlockInfo;
typedef mav1cu_sb_info SbInfo;
typedef mav1cu_lr_unit LrUnit;

// ---- work counters (the counting build, -DMAV1CU_COUNT) ---------------------
// Algorithmic work units per category, added by the kernels where the work
// is done and read through include/mav1cu_count.h. The product library is
// built without them (WORK discards its operands, which have no side
// effects, so no code remains). Units:
//   W_ME_SAD / W_ME_DSAD   full-pel SAD byte pairs, full resolution / decimated planes
//   W_ME_SATD, W_ANA_SATD  4x4 Hadamard SATD units (motion search / analysis)
//   W_QPEL_TAPS            filter taps of the quarter-pel planes (horizontal + vertical)
//   W_ANA_INTER_PX, W_REC_INTER_PX  inter-predicted samples (8-tap horizontal + vertical each)
//   W_ANA_INTRA_PX, W_REC_INTRA_PX  intra-predicted samples
//   W_ANA_CFL              (sample, alpha) SSE terms of the CfL alpha searches
//   W_REC_FWD_MAC          multiply-accumulates of the forward transform's two matrix passes
//   W_REC_QUANT            quantised coefficients
//   W_REC_INV_OPS          inverse transform operations (per 1D N-point pass, 3 log2 N per point)
//   W_LF_TAPS, W_CDEF_TAPS, W_LR_TAPS  filter taps applied by deblocking, CDEF, loop restoration
enum {
  W_ME_SAD, W_ME_DSAD, W_ME_SATD, W_QPEL_TAPS, W_ANA_SATD, W_ANA_INTER_PX, W_ANA_INTRA_PX, W_ANA_CFL,
  W_REC_INTER_PX, W_REC_INTRA_PX, W_REC_FWD_MAC, W_REC_QUANT, W_REC_INV_OPS, W_LF_TAPS, W_CDEF_TAPS, W_LR_TAPS,
  W_COUNT
};
#if defined(MAV1CU_COUNT) && defined(__CUDACC__)
static __device__ unsigned long long d_work[W_COUNT];
#define WORK(cat, n) atomicAdd(&d_work[cat], (unsigned long long)(n))
#else
#define WORK(cat, n) ((void)(n))  // discarded (the operands have no side effects)
#endif

// ---- AV1 enumerations (specification section 6.10) -------------------------
enum { INTRA_FRAME = 0, LAST_FRAME = 1, GOLDEN_FRAME = 4, ALTREF_FRAME = 7 };
enum {
  BLOCK_4X4, BLOCK_4X8, BLOCK_8X4, BLOCK_8X8, BLOCK_8X16, BLOCK_16X8, BLOCK_16X16, BLOCK_16X32, BLOCK_32X16,
  BLOCK_32X32, BLOCK_32X64, BLOCK_64X32, BLOCK_64X64, BLOCK_64X128, BLOCK_128X64, BLOCK_128X128, BLOCK_4X16,
  BLOCK_16X4, BLOCK_8X32, BLOCK_32X8, BLOCK_16X64, BLOCK_64X16
};
enum {
  PARTITION_NONE, PARTITION_HORZ, PARTITION_VERT, PARTITION_SPLIT, PARTITION_HORZ_A, PARTITION_HORZ_B,
  PARTITION_VERT_A, PARTITION_VERT_B, PARTITION_HORZ_4, PARTITION_VERT_4
};
enum {
  DC_PRED, V_PRED, H_PRED, D45_PRED, D135_PRED, D113_PRED, D157_PRED, D203_PRED, D67_PRED, SMOOTH_PRED,
  SMOOTH_V_PRED, SMOOTH_H_PRED, PAETH_PRED, UV_CFL_PRED, NEWMV = 16
};
enum {
  TX_4X4, TX_8X8, TX_16X16, TX_32X32, TX_64X64, TX_4X8, TX_8X4, TX_8X16, TX_16X8, TX_16X32, TX_32X16,
  TX_32X64, TX_64X32, TX_4X16, TX_16X4, TX_8X32, TX_32X8, TX_16X64, TX_64X16
};
enum {
  DCT_DCT, ADST_DCT, DCT_ADST, ADST_ADST, FLIPADST_DCT, DCT_FLIPADST, FLIPADST_FLIPADST, ADST_FLIPADST,
  FLIPADST_ADST, IDTX, V_DCT, H_DCT, V_ADST, H_ADST, V_FLIPADST, H_FLIPADST
};
enum { TX_SET_DCTONLY = 0, TX_SET_INTRA_1 = 1, TX_SET_INTRA_2 = 2, TX_SET_INTER_1 = 1, TX_SET_INTER_2 = 2,
       TX_SET_INTER_3 = 3 };
enum { EIGHTTAP = 0, EIGHTTAP_SMOOTH = 1, EIGHTTAP_SHARP = 2 };
enum { RESTORE_NONE = 0, RESTORE_WIENER = 1, RESTORE_SGRPROJ = 2, RESTORE_SWITCHABLE = 3 };

#define MAX_LOOP_FILTER 63
#define MAX_TX_DEPTH 2
#define MAX_ANGLE_DELTA 3
#define ANGLE_STEP 3
#define MI_SIZE 4
#define SUBPEL_MASK 15
#define FILTER_BITS 7
#define SGRPROJ_RST_BITS 4
#define SGRPROJ_PRJ_BITS 7
#define SGRPROJ_MTABLE_BITS 20
#define SGRPROJ_RECIP_BITS 12
#define SGRPROJ_SGR_BITS 8

// Superblock layout of the analysis / motion-search tables: square nodes
// 64x64 (1), 32x32 (4), 16x16 (16), 8x8 (64) in raster order per level.
#define NUM_NODES 85
#define MAX_BLOCKS_PER_SB 64
#define COEFS_PER_SB 6144
#define A_SLOTS 13
#define A_ITEMS (NUM_NODES * A_SLOTS)
HD int node_base(int level) { return level == 0 ? 0 : level == 1 ? 1 : level == 2 ? 5 : 21; }
HD int level_bsize(int l) { return l == 0 ? BLOCK_64X64 : l == 1 ? BLOCK_32X32 : l == 2 ? BLOCK_16X16 : BLOCK_8X8; }

// Turbo mask bits (FrameParams.turbo; reference k_me.h:79-92, k_analysis.h:38-43,598-604).
#define T_SQUARE 1
#define T_ME_CR1 2
#define T_ME_L3COPY 4
#define T_ME_KEEP 8
#define T_ME_HPEL 16
#define T_ME_DEC 32
#define T_ME_CR2 64
#define T_INTRA 128
#define T_KEY_SQUARE 256
#define T_ME_REF2 512
#define T_LEAF_NO8 1024
#define T_ME_L3SUB 4096
#define T_ME_CROSS 8192
#define T_ME_G3COPY 16384
#define T_ME_HALF01 32768
#define T_ME_RSUB 65536
#define T_ME_HME3 131072
#define T_ME_USUB 262144
#define T_ANA_USUB 4194304

// ---- tables ------------------------------------------------------------------
// Small tables read with warp-uniform indices live in constant memory; tables
// indexed per thread (scans, filters) live in global memory (L1-cached).
#define MAV1_TABLES(X)                                                                  \
  X(__constant__, Cos128_Lookup) X(__constant__, Transform_Row_Shift)                   \
  X(__constant__, Tx_Width) X(__constant__, Tx_Height) X(__constant__, Tx_Width_Log2)   \
  X(__constant__, Tx_Height_Log2) X(__constant__, Tx_Size_Sqr)                          \
  X(__constant__, Tx_Size_Sqr_Up) X(__constant__, Split_Tx_Size)                        \
  X(__constant__, Mode_To_Txfm) X(__constant__, Tx_Type_In_Set_Intra)                   \
  X(__constant__, Tx_Type_In_Set_Inter) X(__constant__, Max_Tx_Size_Rect)               \
  X(__constant__, Max_Tx_Depth) X(__constant__, Num_4x4_Blocks_Wide)                    \
  X(__constant__, Num_4x4_Blocks_High) X(__constant__, Mi_Width_Log2)                   \
  X(__constant__, Mi_Height_Log2) X(__constant__, Subsampled_Size)                      \
  X(__constant__, Partition_Subsize) X(__constant__, Mode_To_Angle)                     \
  X(__constant__, Intra_Edge_Kernel) X(__constant__, Div_Table)                         \
  X(__constant__, Cdef_Uv_Dir) X(__constant__, Cdef_Pri_Taps)                           \
  X(__constant__, Cdef_Sec_Taps) X(__constant__, Cdef_Directions)                       \
  X(__constant__, Sgr_Params) X(__constant__, Wiener_Taps_Min)                          \
  X(__constant__, Wiener_Taps_Max) X(__constant__, Wiener_Taps_K)                       \
  X(__constant__, Wiener_Taps_Mid) X(__constant__, Sgrproj_Xqd_Min)                     \
  X(__constant__, Sgrproj_Xqd_Max) X(__constant__, Sgrproj_Xqd_Mid)                     \
  X(__device__, Subpel_Filters) X(__device__, Dr_Intra_Derivative)                      \
  X(__device__, Sm_Weights_Tx_4x4) X(__device__, Sm_Weights_Tx_8x8)                     \
  X(__device__, Sm_Weights_Tx_16x16) X(__device__, Sm_Weights_Tx_32x32)                 \
  X(__device__, Sm_Weights_Tx_64x64)

// One copy per translation unit (the library is a single one): device copies
// in constant / global memory, host copies for the host helpers.
#if defined(__CUDACC__)
#define MAV1_DEF_DTABLE(space, name) static space const int32_t d_##name MAV1T_##name##_DIMS = MAV1T_##name;
MAV1_TABLES(MAV1_DEF_DTABLE)
#endif
#define MAV1_DEF_HTABLE(space, name) static const int32_t h_##name MAV1T_##name##_DIMS = MAV1T_##name;
MAV1_TABLES(MAV1_DEF_HTABLE)
static const int32_t h_Dc_Qlookup MAV1T_Dc_Qlookup_DIMS = MAV1T_Dc_Qlookup;
static const int32_t h_Ac_Qlookup MAV1T_Ac_Qlookup_DIMS = MAV1T_Ac_Qlookup;

#if defined(__CUDA_ARCH__)
#define T(name) d_##name
#else
#define T(name) h_##name
#endif

// ---- integer helpers (AV1 specification section 4.7) -------------------------
HD int imin(int a, int b) { return a < b ? a : b; }
HD int imax(int a, int b) { return a > b ? a : b; }
HD int iabs(int a) { return a < 0 ? -a : a; }
HD int clip3(int lo, int hi, int x) { return x < lo ? lo : (x > hi ? hi : x); }
HD int clip1(int x) { return clip3(0, 255, x); }
HD int round2(int x, int n) { return n == 0 ? x : ((x + (1 << (n - 1))) >> n); }
HD int64_t round2l(int64_t x, int n) { return n == 0 ? x : ((x + ((int64_t)1 << (n - 1))) >> n); }
HD int round2signed(int x, int n) { return x >= 0 ? round2(x, n) : -round2(-x, n); }
HD int floor_log2(int x) {
  int s = 0;
  while (x > 1) {
    x >>= 1;
    s++;
  }
  return s;
}

// Sample read of a frame written during the same launch by other CTAs: through
// L2 (L1 is not coherent across SMs within a launch).
HD int ldpx(const uint8_t *p) {
#if defined(__CUDA_ARCH__)
  return __ldcg(p);
#else
  return *p;
#endif
}

HD int block_w(int bs) { return 4 * T(Num_4x4_Blocks_Wide)[bs]; }
HD int block_h(int bs) { return 4 * T(Num_4x4_Blocks_High)[bs]; }

// Tile column bounds (uniform spacing, one tile row; k_common.h:89-94).
HD int tile_col_start(const FrameParams *fp, int miCol) { return ((miCol >> 4) / fp->tile_w_sb) * fp->tile_w_sb * 16; }
HD int tile_col_end(const FrameParams *fp, int miCol) {
  return imin(fp->mi_cols, tile_col_start(fp, miCol) + fp->tile_w_sb * 16);
}

// Luma transform size of an intra block at tx_depth (k_common.h:131-135).
HD int depth_tx_size(int bs, int depth) {
  int t = T(Max_Tx_Size_Rect)[bs];
  for (int i = 0; i < depth; i++) t = T(Split_Tx_Size)[t];
  return t;
}

// get_tx_size( ) for chroma (spec 5.11.37).
HD int uv_tx_size(int miSize, int subX, int subY) {
  int uvTx = T(Max_Tx_Size_Rect)[T(Subsampled_Size)[miSize][subX][subY]];
  if (T(Tx_Width)[uvTx] == 64 || T(Tx_Height)[uvTx] == 64) {
    if (T(Tx_Width)[uvTx] == 16) return TX_16X32;
    if (T(Tx_Height)[uvTx] == 16) return TX_32X16;
    return TX_32X32;
  }
  return uvTx;
}

// get_tx_set( ) (spec 5.11.48).
HD int get_tx_set(int txSz, int isInter, int reducedTxSet) {
  int sqr = T(Tx_Size_Sqr)[txSz], sqrUp = T(Tx_Size_Sqr_Up)[txSz];
  if (sqrUp > TX_32X32) return TX_SET_DCTONLY;
  if (isInter) {
    if (reducedTxSet || sqrUp == TX_32X32) return TX_SET_INTER_3;
    if (sqr == TX_16X16) return TX_SET_INTER_2;
    return TX_SET_INTER_1;
  }
  if (sqrUp == TX_32X32) return TX_SET_DCTONLY;
  if (reducedTxSet) return TX_SET_INTRA_2;
  if (sqr == TX_16X16) return TX_SET_INTRA_2;
  return TX_SET_INTRA_1;
}

HD int tx_type_in_set(int set, int t, int isInter) {
  return isInter ? T(Tx_Type_In_Set_Inter)[set][t] : T(Tx_Type_In_Set_Intra)[set][t];
}

// compute_tx_type( ) for a chroma plane (spec 5.11.40).
HD int chroma_tx_type(int txSz, int isInter, int uvMode, int lumaTxType, int reducedTxSet) {
  if (T(Tx_Size_Sqr_Up)[txSz] > TX_32X32) return DCT_DCT;
  int set = get_tx_set(txSz, isInter, reducedTxSet);
  int t = isInter ? lumaTxType : T(Mode_To_Txfm)[uvMode];
  if (!tx_type_in_set(set, t, isInter)) return DCT_DCT;
  return t;
}

// Number of coefficients the decoder scans (spec 5.11.39 segEob).
HD int seg_eob(int txSz) {
  if (txSz == TX_16X64 || txSz == TX_64X16) return 512;
  return imin(1024, T(Tx_Width)[txSz] * T(Tx_Height)[txSz]);
}

// Whether UV_CFL_PRED may be coded (spec 8.3.2 uv_mode cdf selection).
HD int cfl_allowed(int miSize, int lossless) {
  if (lossless) return T(Subsampled_Size)[miSize][1][1] == BLOCK_4X4;
  return imax(block_w(miSize), block_h(miSize)) <= 32;
}

HD int intra_is_directional(int mode) { return mode >= V_PRED && mode <= D67_PRED; }

// Scan order selector (spec 5.11.47 get_scan): index into the scan table set
// uploaded per session (see scan_table_index in session.cu).
enum { SCAN_DEFAULT = 0, SCAN_MROW = 1, SCAN_MCOL = 2 };
HD int scan_kind(int txSz, int planeTxType, int *sizeOut) {
  if (txSz == TX_16X64) { *sizeOut = TX_16X32; return SCAN_DEFAULT; }
  if (txSz == TX_64X16) { *sizeOut = TX_32X16; return SCAN_DEFAULT; }
  if (T(Tx_Size_Sqr_Up)[txSz] == TX_64X64) { *sizeOut = TX_32X32; return SCAN_DEFAULT; }
  *sizeOut = txSz;
  if (planeTxType == IDTX) return SCAN_DEFAULT;
  int preferRow = planeTxType == V_DCT || planeTxType == V_ADST || planeTxType == V_FLIPADST;
  int preferCol = planeTxType == H_DCT || planeTxType == H_ADST || planeTxType == H_FLIPADST;
  // row / column scans exist only up to 16x16 (and 4x16 / 16x4)
  int small = txSz == TX_4X4 || txSz == TX_4X8 || txSz == TX_8X4 || txSz == TX_8X8 || txSz == TX_8X16 ||
              txSz == TX_16X8 || txSz == TX_16X16 || txSz == TX_4X16 || txSz == TX_16X4;
  if (preferRow) return small ? SCAN_MROW : SCAN_DEFAULT;
  if (preferCol) return small ? SCAN_MCOL : SCAN_DEFAULT;
  return SCAN_DEFAULT;
}
