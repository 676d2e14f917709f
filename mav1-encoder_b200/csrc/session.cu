// libmav1cu: the C ABI of include/mav1cu.h over the sm_100a stage kernels.
//
// Single translation unit: the constant tables (tables.inc) and every stage
// (me.cuh, analysis.cuh, recon.cuh, filters.cuh) are compiled here so the
// tables exist once per device image.
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <memory>
#include <mutex>
#include <vector>

#include "common.cuh"
#include "tables.inc"
#include "tx.cuh"
#include "pred.cuh"
#include "me.cuh"
#include "analysis.cuh"
#include "recon.cuh"
#include "filters.cuh"
#include "stream.cuh"
#include "export.cuh"
#include "lrsearch.cuh"

// dynamic shared memory of the analysis pass-1 kernel for candidate groups of
// `group` threads: a WarpMem (edge scratch) per group (per warp for CTA groups)
// and one reduction word per warp
#define ANA_SMEM(group) (ana::ana_groups(group) * sizeof(ana::WarpMem) + ANA_THREADS / 32 * sizeof(long long))

namespace {

struct Geometry {
  int w, h, mi_cols, mi_rows, sb_cols, sb_rows, num_sbs;
  int stride[3], plane_h[3], offset[3];
  size_t frame_bytes;
};

Geometry make_geometry(int w, int h) {
  // frame layout of the reference encoder (encoder.c:93-120)
  Geometry g;
  g.w = w;
  g.h = h;
  g.mi_cols = 2 * ((w + 7) >> 3);
  g.mi_rows = 2 * ((h + 7) >> 3);
  g.sb_cols = (g.mi_cols + 15) >> 4;
  g.sb_rows = (g.mi_rows + 15) >> 4;
  g.num_sbs = g.sb_cols * g.sb_rows;
  g.stride[0] = g.sb_cols * 64;
  g.stride[1] = g.stride[2] = g.sb_cols * 32;
  g.plane_h[0] = g.sb_rows * 64;
  g.plane_h[1] = g.plane_h[2] = g.sb_rows * 32;
  g.offset[0] = 0;
  g.offset[1] = g.stride[0] * g.plane_h[0];
  g.offset[2] = g.offset[1] + g.stride[1] * g.plane_h[1];
  g.frame_bytes = (size_t)g.offset[2] + (size_t)g.stride[2] * g.plane_h[2];
  return g;
}

}  // namespace

// exports whose completion a host consumer can wait for individually
#define XRING 64

struct mav1cu_session {
  Geometry g;
  int max_presets;
  cudaStream_t stream, own_stream;
  void *buf[MAV1CU_BUF_COUNT];
  size_t size[MAV1CU_BUF_COUNT];
  // internal device state
  uint8_t *qp[2];          // 16 quarter-pel planes per reference
  uint8_t *dsrc, *dref[2]; // decimated planes
  // planes of the references supplied by a stream for the next motion
  // search (its per-picture cache); null: the search builds its own
  const uint8_t *ext_qp[2], *ext_dref[2];
  uint8_t *ys, *uvs;       // edge-type marks per mi
  int32_t *mats_t;         // MATS with every matrix transposed (row passes read it along the output index)
  int mats_dirty;          // MATS changed since mats_t was derived
  int mats_exposed;        // MATS's device address was handed out: derive mats_t before every recon
  int *waves;              // superblocks in wave order
  int *status;             // device status: [0] error, [1] abort, [2] queue head, [3] intra blocks, [4] queue tail
  int *blk_at;             // block index per 4x4 luma unit
  int *blk_list;           // recon claim list
  int *blk_done;           // per-block completion flags of the recon launch: luma, then chroma
  int *dep_count, *succ_count, *succ, *queue, *corners;  // intra ready queue and corner bits (rec::Ctx)
  int resident_recon;      // intra recon workers (CTAs, one per SM)
  int4 *xcounts;           // compact export: per-superblock counts, block and level bases, zero run / fit flag
  int *xblk_base, *xcoef_base, *xmeta;
  void *ximage;            // session-owned export image (page-locked, mapped), allocated on first request
  int xseq;                // exports enqueued
  cudaStream_t xs;         // transfer stream the exports run on, forked from `stream`
  cudaEvent_t x_fork, x_done;
  int x_pending;           // an export may still read the session's buffers: writers wait for x_done
  cudaEvent_t xring[XRING];  // completion of export seq, recorded at xring[seq % XRING] (blocking sync)
  int device;              // the device the session's memory lives on
  cudaStream_t ss;         // status reads of host consumers (never waits for the session's other streams)
  lrs::Fit *lrfit;         // loop-restoration search: first-pass results per restoration unit
  int *lr_types;           // the search's lr_type per plane (exported with the frame)
  int max_lr_units;
  int lr_searched;         // the current frame's LR units and types come from mav1cu_lr_search
  int64_t device_bytes;    // device memory this session allocated
  int fault_hold, fault_spins;  // failure-detection test: the next recon's held block and poll limit
  std::vector<int> wave_start, wave_len;
  int wave_tile_w;
  FrameParams fp;          // host copy of the current parameters
  int have_params;
  int64_t launches;
  int err;
  char msg[512];
};

static int set_error(mav1cu_session *s, int code, const char *fmt, ...) {
  if (!s->err) {
    s->err = code;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(s->msg, sizeof s->msg, fmt, ap);
    va_end(ap);
  }
  return s->err;
}

static int check_cuda(mav1cu_session *s, cudaError_t e, const char *what) {
  if (e != cudaSuccess) return set_error(s, MAV1CU_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return MAV1CU_OK;
}

static int after_launch(mav1cu_session *s, const char *what) {
  s->launches++;
  return check_cuda(s, cudaGetLastError(), what);
}

// Work that overwrites an exported buffer (BLOCKS, SBS, COEFS, CDEF_CHOICE,
// REC) waits until the export reading it, on the transfer stream, is done.
static void export_fence(mav1cu_session *s) {
  if (s->x_pending) {
    cudaStreamWaitEvent(s->stream, s->x_done, 0);
    s->x_pending = 0;
  }
}

// ---- inverse scan tables ------------------------------------------------------------

// Scan table of (txSz, type) exactly as the reference selects it (get_scan
// and its per-size fallbacks, k_scan.h:241-292).
static const int32_t *host_scan(int txSz, int t, int *len) {
  if (txSz == TX_16X64) { *len = 512; return h_Default_Scan_16x32; }
  if (txSz == TX_64X16) { *len = 512; return h_Default_Scan_32x16; }
  if (h_Tx_Size_Sqr_Up[txSz] == TX_64X64) { *len = 1024; return h_Default_Scan_32x32; }
  int preferRow = t == V_DCT || t == V_ADST || t == V_FLIPADST;
  int preferCol = t == H_DCT || t == H_ADST || t == H_FLIPADST;
  if (t == IDTX) preferRow = preferCol = 0;
#define SZ(tx, name, n) if (txSz == tx) { *len = n; return h_##name; }
  if (preferRow) {
    SZ(TX_4X4, Mrow_Scan_4x4, 16) SZ(TX_4X8, Mrow_Scan_4x8, 32) SZ(TX_8X4, Mrow_Scan_8x4, 32)
    SZ(TX_8X8, Mrow_Scan_8x8, 64) SZ(TX_8X16, Mrow_Scan_8x16, 128) SZ(TX_16X8, Mrow_Scan_16x8, 128)
    SZ(TX_16X16, Mrow_Scan_16x16, 256) SZ(TX_4X16, Mrow_Scan_4x16, 64)
    *len = 64;
    return h_Mrow_Scan_16x4;
  }
  if (preferCol) {
    SZ(TX_4X4, Mcol_Scan_4x4, 16) SZ(TX_4X8, Mcol_Scan_4x8, 32) SZ(TX_8X4, Mcol_Scan_8x4, 32)
    SZ(TX_8X8, Mcol_Scan_8x8, 64) SZ(TX_8X16, Mcol_Scan_8x16, 128) SZ(TX_16X8, Mcol_Scan_16x8, 128)
    SZ(TX_16X16, Mcol_Scan_16x16, 256) SZ(TX_4X16, Mcol_Scan_4x16, 64)
    *len = 64;
    return h_Mcol_Scan_16x4;
  }
  SZ(TX_4X4, Default_Scan_4x4, 16) SZ(TX_4X8, Default_Scan_4x8, 32) SZ(TX_8X4, Default_Scan_8x4, 32)
  SZ(TX_8X8, Default_Scan_8x8, 64) SZ(TX_8X16, Default_Scan_8x16, 128) SZ(TX_16X8, Default_Scan_16x8, 128)
  SZ(TX_16X16, Default_Scan_16x16, 256) SZ(TX_16X32, Default_Scan_16x32, 512)
  SZ(TX_32X16, Default_Scan_32x16, 512) SZ(TX_4X16, Default_Scan_4x16, 64) SZ(TX_16X4, Default_Scan_16x4, 64)
  SZ(TX_8X32, Default_Scan_8x32, 256) SZ(TX_32X8, Default_Scan_32x8, 256)
#undef SZ
  *len = 1024;
  return h_Default_Scan_32x32;
}

static int upload_inverse_scans(mav1cu_session *s) {
  static const int rep[3] = {DCT_DCT, V_DCT, H_DCT};
  std::vector<int16_t> data;
  std::vector<const int32_t *> seen;
  std::vector<int> seenOff;
  int off[3][19];
  for (int k = 0; k < 3; k++)
    for (int t = 0; t < 19; t++) {
      int len;
      const int32_t *sc = host_scan(t, rep[k], &len);
      int found = -1;
      for (size_t i = 0; i < seen.size(); i++)
        if (seen[i] == sc) found = seenOff[i];
      if (found < 0) {
        found = (int)data.size();
        seen.push_back(sc);
        seenOff.push_back(found);
        data.resize(data.size() + len);
        for (int c = 0; c < len; c++) data[found + sc[c]] = (int16_t)c;
      }
      off[k][t] = found;
    }
  if (data.size() > 8192) return set_error(s, MAV1CU_ERR_ARG, "inverse scan tables exceed their space");
  if (check_cuda(s, cudaMemcpyToSymbol(rec::d_inv_scan, data.data(), data.size() * sizeof(int16_t)), "scan tables"))
    return s->err;
  return check_cuda(s, cudaMemcpyToSymbol(rec::d_inv_scan_off, off, sizeof off), "scan offsets");
}

// ---- forward matrices (fwd_matrices.c:17-65) ---------------------------------------------

// Matrix of the 1-D inverse kernel `kind` of length n applied to scaled
// impulses, then its least-squares inverse F = (A^T A)^-1 A^T by Gauss-Jordan
// with partial pivoting, rounded to Q20. The double-precision operations and
// their order are those of the reference derivation, so the integer tables
// are identical (checked against the reference's table by the tests).
static void build_fwd_one(int kind, int log2n, int32_t *out) {
  int n = 1 << log2n, m = n > 32 ? 32 : n;
  // working arrays of this call (sessions may be created from several host
  // threads at once)
  std::vector<double> Av(64 * 32), Mv(32 * (32 + 64));
  double(*A)[32] = (double(*)[32])Av.data();
  double(*M)[32 + 64] = (double(*)[32 + 64])Mv.data();
  const double S = 65536.0;
  for (int j = 0; j < m; j++) {
    int32_t t[64];
    for (int i = 0; i < 64; i++) t[i] = 0;
    t[j] = (int32_t)S;
    tx::inverse_1d(t, kind, log2n, 31);
    for (int i = 0; i < n; i++) A[i][j] = t[i] / S;
  }
  for (int r = 0; r < m; r++) {
    for (int c = 0; c < m; c++) {
      double acc = 0;
      for (int i = 0; i < n; i++) acc += A[i][r] * A[i][c];
      M[r][c] = acc;
    }
    for (int i = 0; i < n; i++) M[r][m + i] = A[i][r];
  }
  for (int p = 0; p < m; p++) {
    int best = p;
    for (int r = p + 1; r < m; r++)
      if (fabs(M[r][p]) > fabs(M[best][p])) best = r;
    if (best != p)
      for (int c = 0; c < m + n; c++) {
        double t = M[p][c];
        M[p][c] = M[best][c];
        M[best][c] = t;
      }
    double inv = 1.0 / M[p][p];
    for (int c = 0; c < m + n; c++) M[p][c] *= inv;
    for (int r = 0; r < m; r++) {
      if (r == p || M[r][p] == 0) continue;
      double f = M[r][p];
      for (int c = 0; c < m + n; c++) M[r][c] -= f * M[p][c];
    }
  }
  for (int k = 0; k < m; k++)
    for (int i = 0; i < n; i++) out[k * n + i] = (int32_t)lrint(M[k][m + i] * (double)(1 << 20));
}

static void build_fwd_all(int32_t *mats) {
  memset(mats, 0, sizeof(int32_t) * 4096 * 15);
  for (int kind = 0; kind < 3; kind++)
    for (int log2n = 2; log2n <= 6; log2n++) {
      if (kind == tx::KIND_ADST && log2n > 4) continue;
      if (kind == tx::KIND_IDTX && log2n > 5) continue;
      build_fwd_one(kind, log2n, mats + rec::fwd_slot(kind, log2n));
    }
}

// The table is a constant of the transforms: derived once per process.
extern "C" void mav1cu_build_fwd_matrices(int32_t *mats) {
  static std::vector<int32_t> table(4096 * 15);
  static std::once_flag once;
  std::call_once(once, [] { build_fwd_all(table.data()); });
  memcpy(mats, table.data(), sizeof(int32_t) * 4096 * 15);
}

// ---- session -------------------------------------------------------------------------

static void free_all(mav1cu_session *s) {
  for (int i = 0; i < MAV1CU_BUF_COUNT; i++)
    if (s->buf[i]) cudaFree(s->buf[i]);
  void *extra[] = {s->qp[0], s->qp[1], s->dsrc, s->dref[0], s->dref[1], s->ys, s->uvs, s->waves, s->status, s->blk_at, s->blk_list,
                   s->blk_done, s->mats_t, s->dep_count, s->succ_count, s->succ, s->queue, s->corners,
                   s->xcounts, s->xblk_base, s->xcoef_base, s->xmeta, s->lrfit, s->lr_types};
  for (void *p : extra)
    if (p) cudaFree(p);
  if (s->ximage) cudaFreeHost(s->ximage);
  if (s->x_fork) cudaEventDestroy(s->x_fork);
  if (s->x_done) cudaEventDestroy(s->x_done);
  for (int i = 0; i < XRING; i++)
    if (s->xring[i]) cudaEventDestroy(s->xring[i]);
  if (s->xs) cudaStreamDestroy(s->xs);
  if (s->ss) cudaStreamDestroy(s->ss);
  if (s->own_stream) cudaStreamDestroy(s->own_stream);
}

// Device allocation counted into the session's footprint.
static cudaError_t dmalloc(mav1cu_session *s, void **p, size_t bytes) {
  cudaError_t e = cudaMalloc(p, bytes);
  if (e == cudaSuccess) s->device_bytes += (int64_t)bytes;
  return e;
}

// The device bytes mav1cu_session_create allocates for this geometry: the
// same list of allocations, summed (checked against the count of a real
// session by the GPU tests).
static int64_t session_bytes(const Geometry &g, int maxPresets) {
  size_t fb = g.frame_bytes, nsb = (size_t)g.num_sbs, mi = (size_t)g.mi_rows * g.mi_cols;
  size_t plane = (size_t)g.w * g.h, dplane = (size_t)((g.w + 3) >> 2) * ((g.h + 3) >> 2);
  size_t nblk = (size_t)MAX_BLOCKS_PER_SB * nsb;
  size_t lrUnits = 3 * (size_t)(g.sb_rows + 1) * (g.sb_cols + 1);
  size_t b = 6 * fb;                                                   // SRC REC REF GOLD DBK LROUT
  b += sizeof(FrameParams) + sizeof(int32_t) * 4096 * 15;             // PARAMS MATS
  b += 2 * sizeof(int32_t) * 2 * NUM_NODES * nsb;                      // MVFIELD MVGOLD
  b += sizeof(BlockInfo) * MAX_BLOCKS_PER_SB * nsb + sizeof(SbInfo) * nsb + sizeof(int32_t) * COEFS_PER_SB * nsb;
  b += mi + fb * (maxPresets ? maxPresets : 1) + nsb;                 // LFMASK CDEFBUF CDEF_CHOICE
  b += sizeof(LrUnit) * lrUnits;                                       // LRUNITS
  b += (sizeof(int64_t) + sizeof(BlockInfo)) * A_ITEMS * nsb;          // ACOSTS AINFOS
  b += 2 * 16 * plane + 3 * dplane + 2 * mi;                           // quarter-pel, decimated, edge marks
  b += sizeof(int) * (nsb + 8 + mi) + sizeof(int32_t) * 4096 * 15;     // waves, status, block map, mats_t
  b += sizeof(int) * nblk * (4 + MAX_SUCC);                            // ready queue state
  b += sizeof(int) * MAX_BLOCKS_PER_SB * nsb * 3;                      // claim list, completion flags
  b += sizeof(int4) * nsb + 2 * sizeof(int) * nsb + sizeof(int) * 4;   // export scratch
  b += sizeof(lrs::Fit) * lrUnits + sizeof(int) * 4;                   // LR search
  return (int64_t)b;
}

extern "C" int64_t mav1cu_session_device_bytes(const mav1cu_session *s) { return s->device_bytes; }

extern "C" int mav1cu_session_create(int width, int height, int max_cdef_presets, mav1cu_session **out, char *err,
                                     size_t errlen) {
  *out = NULL;
  if (width < 16 || height < 16 || width > 65536 || height > 65536 || max_cdef_presets < 0 || max_cdef_presets > 4) {
    snprintf(err, errlen, "unsupported session %dx%d (%d CDEF presets)", width, height, max_cdef_presets);
    return MAV1CU_ERR_ARG;
  }
  mav1cu_session *s = new mav1cu_session();
  s->g = make_geometry(width, height);
  s->max_presets = max_cdef_presets;
  const Geometry &g = s->g;
  size_t fb = g.frame_bytes, nsb = (size_t)g.num_sbs;
  s->size[MAV1CU_BUF_SRC] = s->size[MAV1CU_BUF_REC] = s->size[MAV1CU_BUF_REF] = s->size[MAV1CU_BUF_GOLD] = fb;
  s->size[MAV1CU_BUF_DBK] = s->size[MAV1CU_BUF_LROUT] = fb;
  s->size[MAV1CU_BUF_PARAMS] = sizeof(FrameParams);
  s->size[MAV1CU_BUF_MATS] = sizeof(int32_t) * 4096 * 15;
  s->size[MAV1CU_BUF_MVFIELD] = s->size[MAV1CU_BUF_MVGOLD] = sizeof(int32_t) * 2 * NUM_NODES * nsb;
  s->size[MAV1CU_BUF_BLOCKS] = sizeof(BlockInfo) * MAX_BLOCKS_PER_SB * nsb;
  s->size[MAV1CU_BUF_SBS] = sizeof(SbInfo) * nsb;
  s->size[MAV1CU_BUF_COEFS] = sizeof(int32_t) * COEFS_PER_SB * nsb;
  s->size[MAV1CU_BUF_LFMASK] = (size_t)g.mi_rows * g.mi_cols;
  s->size[MAV1CU_BUF_CDEFBUF] = fb * (max_cdef_presets ? max_cdef_presets : 1);
  s->size[MAV1CU_BUF_CDEF_CHOICE] = nsb;
  s->size[MAV1CU_BUF_LRUNITS] = sizeof(LrUnit) * 3 * (size_t)(g.sb_rows + 1) * (g.sb_cols + 1);
  s->size[MAV1CU_BUF_ACOSTS] = sizeof(int64_t) * A_ITEMS * nsb;
  s->size[MAV1CU_BUF_AINFOS] = sizeof(BlockInfo) * A_ITEMS * nsb;
  cudaError_t e = cudaSuccess;
  for (int i = 0; i < MAV1CU_BUF_COUNT && e == cudaSuccess; i++) {
    e = dmalloc(s, (void **)&s->buf[i], s->size[i]);
    if (e == cudaSuccess) e = cudaMemset(s->buf[i], 0, s->size[i]);
  }
  size_t plane = (size_t)width * height, dplane = (size_t)((width + 3) >> 2) * ((height + 3) >> 2);
  if (e == cudaSuccess) e = dmalloc(s, (void **)&s->qp[0], 16 * plane);
  if (e == cudaSuccess) e = dmalloc(s, (void **)&s->qp[1], 16 * plane);
  if (e == cudaSuccess) e = dmalloc(s, (void **)&s->dsrc, dplane);
  if (e == cudaSuccess) e = dmalloc(s, (void **)&s->dref[0], dplane);
  if (e == cudaSuccess) e = dmalloc(s, (void **)&s->dref[1], dplane);
  if (e == cudaSuccess) e = dmalloc(s, (void **)&s->ys, (size_t)g.mi_rows * g.mi_cols);
  if (e == cudaSuccess) e = dmalloc(s, (void **)&s->uvs, (size_t)g.mi_rows * g.mi_cols);
  if (e == cudaSuccess) e = dmalloc(s, (void **)&s->waves, sizeof(int) * nsb);
  if (e == cudaSuccess) e = dmalloc(s, (void **)&s->status, sizeof(int) * 8);
  if (e == cudaSuccess) e = dmalloc(s, (void **)&s->blk_at, sizeof(int) * g.mi_rows * g.mi_cols);
  if (e == cudaSuccess) e = dmalloc(s, (void **)&s->mats_t, sizeof(int32_t) * 4096 * 15);
  size_t nblk = MAX_BLOCKS_PER_SB * nsb;
  if (e == cudaSuccess) e = dmalloc(s, (void **)&s->dep_count, sizeof(int) * nblk);
  if (e == cudaSuccess) e = dmalloc(s, (void **)&s->succ_count, sizeof(int) * nblk);
  if (e == cudaSuccess) e = dmalloc(s, (void **)&s->succ, sizeof(int) * nblk * MAX_SUCC);
  if (e == cudaSuccess) e = dmalloc(s, (void **)&s->queue, sizeof(int) * nblk);
  if (e == cudaSuccess) e = dmalloc(s, (void **)&s->corners, sizeof(int) * nblk);
  s->mats_dirty = 1;
  if (e == cudaSuccess) e = dmalloc(s, (void **)&s->blk_list, sizeof(int) * MAX_BLOCKS_PER_SB * nsb);
  if (e == cudaSuccess) e = dmalloc(s, (void **)&s->blk_done, 2 * sizeof(int) * MAX_BLOCKS_PER_SB * nsb);
  if (e == cudaSuccess) e = dmalloc(s, (void **)&s->xcounts, sizeof(int4) * nsb);
  if (e == cudaSuccess) e = dmalloc(s, (void **)&s->xblk_base, sizeof(int) * nsb);
  if (e == cudaSuccess) e = dmalloc(s, (void **)&s->xcoef_base, sizeof(int) * nsb);
  if (e == cudaSuccess) e = dmalloc(s, (void **)&s->xmeta, sizeof(int) * 4);
  s->max_lr_units = 3 * (g.sb_rows + 1) * (g.sb_cols + 1);
  if (e == cudaSuccess) e = dmalloc(s, (void **)&s->lrfit, sizeof(lrs::Fit) * s->max_lr_units);
  if (e == cudaSuccess) e = dmalloc(s, (void **)&s->lr_types, sizeof(int) * 4);
  if (e == cudaSuccess) e = cudaMemset(s->lr_types, 0, sizeof(int) * 4);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->own_stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->xs, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->x_fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->x_done, cudaEventDisableTiming);
  for (int i = 0; i < XRING && e == cudaSuccess; i++)
    e = cudaEventCreateWithFlags(&s->xring[i], cudaEventDisableTiming | cudaEventBlockingSync);
  if (e == cudaSuccess) e = cudaGetDevice(&s->device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->ss, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    snprintf(err, errlen, "device allocation failed: %s", cudaGetErrorString(e));
    free_all(s);
    delete s;
    return e == cudaErrorMemoryAllocation ? MAV1CU_ERR_NOMEM : MAV1CU_ERR_CUDA;
  }
  s->stream = s->own_stream;
  cudaMemset(s->status, 0, sizeof(int) * 8);
  cudaMemset(s->blk_at, 0xff, sizeof(int) * g.mi_rows * g.mi_cols);  // -1: no block
  std::vector<int32_t> mats(4096 * 15);
  mav1cu_build_fwd_matrices(mats.data());
  cudaMemcpy(s->buf[MAV1CU_BUF_MATS], mats.data(), mats.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
  if (upload_inverse_scans(s) || check_cuda(s, cudaDeviceSynchronize(), "session setup")) {
    snprintf(err, errlen, "%s", s->msg);
    int code = s->err;
    mav1cu_session_destroy(s);
    return code;
  }
  cudaFuncSetAttribute(rec::k_recon_blocks, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rec::SMEM_INTRA);
  cudaFuncSetAttribute(rec::k_recon_inter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rec::SMEM_INTER);
  {
    int dev = 0, sms = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, rec::k_recon_blocks, rec::INTRA_THREADS, rec::SMEM_INTRA);
    // at most one worker per SM (the kernel keeps max(8, intra blocks / 8) of
    // them): the ready queue keeps them on ready blocks, and the rest of each
    // SM stays free for the other engines' kernels
    s->resident_recon = imax(1, sms * imin(1, imax(1, per)));
  }
  cudaFuncSetAttribute(ana::k_analyze_level, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ANA_SMEM(16));
  cudaFuncSetAttribute(lrs::k_lr_fit, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(lrs::Shared));
  cudaFuncSetAttribute(lrs::k_lr_select, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(lrs::Shared));
  cudaFuncSetAttribute(lrs::k_lr_spec, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(lrs::Shared));
  *out = s;
  return MAV1CU_OK;
}

extern "C" void mav1cu_session_destroy(mav1cu_session *s) {
  if (!s) return;
  cudaStreamSynchronize(s->stream);
  if (s->xs) cudaStreamSynchronize(s->xs);
  free_all(s);
  delete s;
}

extern "C" int mav1cu_set_stream(mav1cu_session *s, void *stream) {
  s->stream = stream ? (cudaStream_t)stream : s->own_stream;
  return MAV1CU_OK;
}
extern "C" void *mav1cu_get_stream(mav1cu_session *s) { return (void *)s->stream; }

extern "C" size_t mav1cu_buf_size(const mav1cu_session *s, int buf) {
  return buf >= 0 && buf < MAV1CU_BUF_COUNT ? s->size[buf] : 0;
}
extern "C" void *mav1cu_buf_device(mav1cu_session *s, int buf) {
  if (buf == MAV1CU_BUF_MATS) s->mats_exposed = 1;
  return buf >= 0 && buf < MAV1CU_BUF_COUNT ? s->buf[buf] : NULL;
}

extern "C" int mav1cu_upload(mav1cu_session *s, int buf, const void *host, size_t bytes) {
  if (s->err) return s->err;
  if (buf < 0 || buf >= MAV1CU_BUF_COUNT || bytes > s->size[buf])
    return set_error(s, MAV1CU_ERR_ARG, "upload: buffer %d, %zu bytes", buf, bytes);
  if (buf == MAV1CU_BUF_MATS) s->mats_dirty = 1;
  export_fence(s);
  return check_cuda(s, cudaMemcpyAsync(s->buf[buf], host, bytes, cudaMemcpyHostToDevice, s->stream), "upload");
}

extern "C" int mav1cu_download(mav1cu_session *s, int buf, void *host, size_t bytes) {
  if (s->err) return s->err;
  if (buf < 0 || buf >= MAV1CU_BUF_COUNT || bytes > s->size[buf])
    return set_error(s, MAV1CU_ERR_ARG, "download: buffer %d, %zu bytes", buf, bytes);
  return check_cuda(s, cudaMemcpyAsync(host, s->buf[buf], bytes, cudaMemcpyDeviceToHost, s->stream), "download");
}

extern "C" int mav1cu_copy(mav1cu_session *s, int dst, int src, size_t bytes) {
  if (s->err) return s->err;
  if (dst < 0 || dst >= MAV1CU_BUF_COUNT || src < 0 || src >= MAV1CU_BUF_COUNT || bytes > s->size[dst] ||
      bytes > s->size[src])
    return set_error(s, MAV1CU_ERR_ARG, "copy: buffers %d <- %d, %zu bytes", dst, src, bytes);
  export_fence(s);
  if (dst == MAV1CU_BUF_MATS) s->mats_dirty = 1;
  return check_cuda(s, cudaMemcpyAsync(s->buf[dst], s->buf[src], bytes, cudaMemcpyDeviceToDevice, s->stream), "copy");
}

// Superblocks in wave order: wave (c - tileStart) + 2r holds the superblocks
// whose left, above-left, above and above-right neighbours (same tile
// column) are in earlier waves. The recon claim list follows this order.
static int build_waves(mav1cu_session *s, int tile_w_sb) {
  const Geometry &g = s->g;
  int nw = tile_w_sb + 2 * (g.sb_rows - 1);
  std::vector<int> list;
  s->wave_start.assign(nw, 0);
  s->wave_len.assign(nw, 0);
  for (int w = 0; w < nw; w++) {
    s->wave_start[w] = (int)list.size();
    for (int r = 0; r < g.sb_rows; r++)
      for (int c = 0; c < g.sb_cols; c++)
        if ((c % tile_w_sb) + 2 * r == w) list.push_back(r * g.sb_cols + c);
    s->wave_len[w] = (int)list.size() - s->wave_start[w];
  }
  s->wave_tile_w = tile_w_sb;
  // in the session's stream order: a plain cudaMemcpy from pageable memory
  // may return before the data lands, and the stream's kernels (non-blocking
  // stream) would not wait for it; the async copy stages the list before it
  // returns
  return check_cuda(s, cudaMemcpyAsync(s->waves, list.data(), list.size() * sizeof(int), cudaMemcpyHostToDevice,
                                       s->stream),
                    "waves");
}

extern "C" int mav1cu_set_params(mav1cu_session *s, const mav1cu_frame_params *fp) {
  if (s->err) return s->err;
  const Geometry &g = s->g;
  if (fp->mi_cols != g.mi_cols || fp->mi_rows != g.mi_rows || fp->frame_w != g.w || fp->frame_h != g.h ||
      fp->stride[0] != g.stride[0] || fp->offset[1] != g.offset[1] || fp->tile_w_sb < 1)
    return set_error(s, MAV1CU_ERR_ARG, "frame parameters do not match the session geometry");
  s->fp = *fp;
  s->have_params = 1;
  s->lr_searched = 0;
  if (s->wave_tile_w != fp->tile_w_sb && build_waves(s, fp->tile_w_sb)) return s->err;
  // by value through a launch: asynchronous for any caller memory (a copy
  // from pageable memory may wait for the stream's earlier work)
  drv::k_store_params<<<1, 128, 0, s->stream>>>(*fp, (FrameParams *)s->buf[MAV1CU_BUF_PARAMS]);
  return after_launch(s, "frame parameters");
}

static int need_params(mav1cu_session *s) {
  if (s->err) return s->err;
  if (!s->have_params) return set_error(s, MAV1CU_ERR_ARG, "stage called before mav1cu_set_params");
  return MAV1CU_OK;
}

#define DP(s) ((const FrameParams *)(s)->buf[MAV1CU_BUF_PARAMS])
#define U8(s, b) ((uint8_t *)(s)->buf[b])

// The motion search's planes of one reference picture (padded layout) on
// the session's stream: the 16 quarter-pel planes and, in the T_ME_DEC mode,
// the decimated plane.
static int build_ref_planes(mav1cu_session *s, const uint8_t *ref, uint8_t *qp, uint8_t *dref) {
  const FrameParams &fp = s->fp;
  dim3 qgrid((fp.frame_w + me::QP_TW - 1) / me::QP_TW, (fp.frame_h + me::QP_TH - 1) / me::QP_TH);
  me::k_qpel_planes<<<qgrid, me::QP_THREADS, 0, s->stream>>>(DP(s), ref, qp);
  if (after_launch(s, "qpel planes")) return s->err;
  if (fp.turbo & T_ME_DEC) {
    int dw = (fp.frame_w + 3) >> 2, dh = (fp.frame_h + 3) >> 2;
    me::k_dec_plane<<<dim3((dw + 127) / 128, dh), 128, 0, s->stream>>>(DP(s), ref, dref);
    if (after_launch(s, "decimated reference")) return s->err;
  }
  return MAV1CU_OK;
}

extern "C" int mav1cu_motion_search(mav1cu_session *s) {
  if (need_params(s)) return s->err;
  const FrameParams &fp = s->fp;
  int nref = fp.golden ? 2 : 1;
  const uint8_t *refs[2] = {U8(s, MAV1CU_BUF_REF), U8(s, MAV1CU_BUF_GOLD)};
  const uint8_t *qp[2] = {s->qp[0], s->qp[1]}, *dref[2] = {s->dref[0], s->dref[1]};
  if (fp.turbo & T_ME_HPEL) {
    for (int r = 0; r < nref; r++) {
      if (s->ext_qp[r]) {  // supplied by the stream's plane cache, complete in stream order
        qp[r] = s->ext_qp[r];
        dref[r] = s->ext_dref[r];
      } else if (build_ref_planes(s, refs[r], s->qp[r], s->dref[r])) {
        return s->err;
      }
    }
    if (fp.turbo & T_ME_DEC) {
      int dw = (fp.frame_w + 3) >> 2, dh = (fp.frame_h + 3) >> 2;
      me::k_dec_plane<<<dim3((dw + 127) / 128, dh), 128, 0, s->stream>>>(DP(s), U8(s, MAV1CU_BUF_SRC), s->dsrc);
      if (after_launch(s, "decimated source")) return s->err;
    }
  }
  for (int r = 0; r < 2; r++) s->ext_qp[r] = s->ext_dref[r] = nullptr;
  me::Frame f[2];
  for (int r = 0; r < 2; r++) {
    f[r].fp = DP(s);
    f[r].src = U8(s, MAV1CU_BUF_SRC);
    f[r].ref = refs[r];
    f[r].qp = qp[r];
    f[r].dsrc = s->dsrc;
    f[r].dref = dref[r];
    f[r].mv = (int32_t *)s->buf[r ? MAV1CU_BUF_MVGOLD : MAV1CU_BUF_MVFIELD];
    f[r].isGold = r;
  }
  for (int level = 0; level < 4; level++) {
    int nodes = s->g.num_sbs << (2 * level);
    // threads per node: the CTA for the 64x64 nodes, half a warp for the 8x8
    // nodes, a warp otherwise
    int group = level == 0 ? 128 : level == 3 ? 16 : 32;
    dim3 grid((nodes + 128 / group - 1) / (128 / group), nref);
    me::k_me_level<<<grid, 128, 0, s->stream>>>(f[0], f[1], level, group);
    if (after_launch(s, "motion search")) return s->err;
  }
  return MAV1CU_OK;
}

static ana::Ctx ana_ctx(mav1cu_session *s) {
  ana::Ctx c;
  c.fp = DP(s);
  c.src = U8(s, MAV1CU_BUF_SRC);
  c.ref = U8(s, MAV1CU_BUF_REF);
  c.gold = U8(s, MAV1CU_BUF_GOLD);
  c.mv = (const int32_t *)s->buf[MAV1CU_BUF_MVFIELD];
  c.mvg = (const int32_t *)s->buf[MAV1CU_BUF_MVGOLD];
  c.costs = (int64_t *)s->buf[MAV1CU_BUF_ACOSTS];
  c.infos = (BlockInfo *)s->buf[MAV1CU_BUF_AINFOS];
  c.blocks = (BlockInfo *)s->buf[MAV1CU_BUF_BLOCKS];
  c.sbs = (SbInfo *)s->buf[MAV1CU_BUF_SBS];
  return c;
}

extern "C" int mav1cu_analyze(mav1cu_session *s) {
  if (need_params(s)) return s->err;
  export_fence(s);
  ana::Ctx c = ana_ctx(s);
  for (int level = 0; level < 4; level++) {
    int slots = ana::level_slots(&s->fp, level);
    long long items = (long long)s->g.num_sbs * (1 << (2 * level)) * slots;
    // threads per candidate: the CTA for 64x64, a warp for 32x32, half a warp
    // for 16x16 and 8x8 (at most 16 luma 4x4 units per candidate)
    int group = level == 0 ? ANA_THREADS : level >= 2 ? 16 : 32, per = ANA_THREADS / group;
    unsigned grid = (unsigned)((items + per - 1) / per);
    ana::k_analyze_level<<<grid, ANA_THREADS, ANA_SMEM(group), s->stream>>>(c, level, slots, group);
    if (after_launch(s, "analysis pass 1")) return s->err;
  }
  ana::k_analyze_table<<<(s->g.num_sbs + TABLE_WARPS - 1) / TABLE_WARPS, 32 * TABLE_WARPS, 0, s->stream>>>(c);
  return after_launch(s, "analysis pass 2");
}

extern "C" int mav1cu_edge_types(mav1cu_session *s) {
  if (need_params(s)) return s->err;
  export_fence(s);
  BlockInfo *blocks = (BlockInfo *)s->buf[MAV1CU_BUF_BLOCKS];
  const SbInfo *sbs = (const SbInfo *)s->buf[MAV1CU_BUF_SBS];
  ana::k_edge_marks<<<s->g.num_sbs, 64, 0, s->stream>>>(DP(s), blocks, sbs, s->ys, s->uvs);
  if (after_launch(s, "edge marks")) return s->err;
  ana::k_edge_types<<<s->g.num_sbs, 64, 0, s->stream>>>(DP(s), blocks, sbs, s->ys, s->uvs);
  return after_launch(s, "edge types");
}

extern "C" int mav1cu_recon(mav1cu_session *s) {
  if (need_params(s)) return s->err;
  export_fence(s);
  rec::Ctx c;
  c.fp = DP(s);
  c.src = U8(s, MAV1CU_BUF_SRC);
  c.rec = U8(s, MAV1CU_BUF_REC);
  c.ref = U8(s, MAV1CU_BUF_REF);
  c.gold = U8(s, MAV1CU_BUF_GOLD);
  c.blocks = (BlockInfo *)s->buf[MAV1CU_BUF_BLOCKS];
  c.sbs = (const SbInfo *)s->buf[MAV1CU_BUF_SBS];
  c.coefs = (int32_t *)s->buf[MAV1CU_BUF_COEFS];
  c.mats = (const int32_t *)s->buf[MAV1CU_BUF_MATS];
  c.mats_t = s->mats_t;
  if (s->mats_dirty || s->mats_exposed) {
    rec::k_transpose_mats<<<15, 256, 0, s->stream>>>(c.mats, s->mats_t);
    if (after_launch(s, "forward matrices")) return s->err;
    s->mats_dirty = 0;
  }
  c.status = s->status;
  c.blk_at = s->blk_at;
  c.done = s->blk_done;
  c.spin_limit = s->fault_spins > 0 ? s->fault_spins : SPIN_LIMIT;
  c.hold = s->fault_spins > 0 ? s->fault_hold : -1;
  s->fault_spins = 0;
  int nsb = s->g.num_sbs;
  if (check_cuda(s, cudaMemsetAsync(s->blk_done, 0, 2 * sizeof(int) * MAX_BLOCKS_PER_SB * nsb, s->stream),
                 "recon flags"))
    return s->err;
  if (!s->fp.frame_is_intra) {
    rec::k_recon_inter<<<nsb, rec::INTER_THREADS, rec::SMEM_INTER, s->stream>>>(c);
    if (after_launch(s, "recon inter blocks")) return s->err;
  }
  // leaf frames code inter blocks only (the analysis never keeps intra there)
  if (s->fp.leaf && !s->fp.frame_is_intra) return MAV1CU_OK;
  rec::k_block_map<<<(nsb + 3) / 4, 128, 0, s->stream>>>(DP(s), c.blocks, c.sbs, s->blk_at);
  if (after_launch(s, "recon unit map")) return s->err;
  rec::k_block_order<<<1, 1024, 0, s->stream>>>(c.blocks, c.sbs, s->waves, nsb, s->blk_list, s->status + 3);
  if (after_launch(s, "recon claim list")) return s->err;
  size_t nblk = (size_t)MAX_BLOCKS_PER_SB * nsb;
  if (check_cuda(s, cudaMemsetAsync(s->succ_count, 0, sizeof(int) * nblk, s->stream), "recon successors") ||
      check_cuda(s, cudaMemsetAsync(s->queue, 0, sizeof(int) * nblk, s->stream), "recon queue") ||
      check_cuda(s, cudaMemsetAsync(s->status + 2, 0, sizeof(int), s->stream), "recon queue head") ||
      check_cuda(s, cudaMemsetAsync(s->status + 4, 0, sizeof(int), s->stream), "recon queue tail"))
    return s->err;
  c.dep_count = s->dep_count;
  c.succ_count = s->succ_count;
  c.succ = s->succ;
  c.queue = s->queue;
  c.corners = s->corners;
  c.qtail = s->status + 4;
  rec::k_block_deps<<<(unsigned)imin((int)((nblk + 3) / 4), 4 * s->resident_recon), 128, 0, s->stream>>>(
      c, s->blk_list, s->status + 3);
  if (after_launch(s, "recon dependencies")) return s->err;
  rec::Claim q;
  q.list = s->blk_list;
  q.total = s->status + 3;
  q.next = s->status + 2;
  rec::k_recon_blocks<<<s->resident_recon, rec::INTRA_THREADS, rec::SMEM_INTRA, s->stream>>>(c, q);
  return after_launch(s, "recon intra blocks");
}

extern "C" int mav1cu_debug_recon_fault(mav1cu_session *s, int hold_block, int spin_limit) {
  if (spin_limit <= 0 || hold_block < 0 || hold_block >= s->g.num_sbs * MAX_BLOCKS_PER_SB)
    return set_error(s, MAV1CU_ERR_ARG, "recon fault: block %d, limit %d", hold_block, spin_limit);
  s->fault_hold = hold_block;
  s->fault_spins = spin_limit;
  return MAV1CU_OK;
}

// The frame core after the motion search: analysis, edge types, recon.
static int frame_core_after_me(mav1cu_session *s) {
  if (mav1cu_analyze(s)) return s->err;
  if (s->fp.enable_intra_edge_filter && mav1cu_edge_types(s)) return s->err;
  return mav1cu_recon(s);
}

extern "C" int mav1cu_frame_core(mav1cu_session *s) {
  if (need_params(s)) return s->err;
  if (!s->fp.frame_is_intra && mav1cu_motion_search(s)) return s->err;
  return frame_core_after_me(s);
}

extern "C" int mav1cu_filter_info(mav1cu_session *s) {
  if (need_params(s)) return s->err;
  flt::k_filter_info<<<s->g.num_sbs, 64, 0, s->stream>>>(DP(s), (const BlockInfo *)s->buf[MAV1CU_BUF_BLOCKS],
                                                           (const SbInfo *)s->buf[MAV1CU_BUF_SBS],
                                                           U8(s, MAV1CU_BUF_LFMASK));
  return after_launch(s, "filter info");
}

extern "C" int mav1cu_filter(mav1cu_session *s, int num_cdef_presets) {
  if (need_params(s)) return s->err;
  if (num_cdef_presets < 0 || num_cdef_presets > s->max_presets)
    return set_error(s, MAV1CU_ERR_ARG, "filter: %d CDEF presets (session holds %d)", num_cdef_presets, s->max_presets);
  export_fence(s);
  const FrameParams &fp = s->fp;
  if (fp.lf_level[0] || fp.lf_level[1] || fp.lf_level[2] || fp.lf_level[3]) {
    for (int pass = 0; pass < 2; pass++) {
      long long lines = pass == 0 ? fp.mi_rows : fp.mi_cols, n = pass == 0 ? fp.mi_cols : fp.mi_rows;
      long long threads = 3 * lines * n * 4;
      flt::k_deblock<<<(unsigned)((threads + 255) / 256), 256, 0, s->stream>>>(DP(s), U8(s, MAV1CU_BUF_REC),
                                                                               U8(s, MAV1CU_BUF_LFMASK), pass);
      if (after_launch(s, "deblock")) return s->err;
    }
  }
  if (num_cdef_presets > 0) {
    int blocks = ((fp.mi_cols + 1) >> 1) * ((fp.mi_rows + 1) >> 1);
    flt::k_cdef<<<blocks, 64, 0, s->stream>>>(DP(s), U8(s, MAV1CU_BUF_REC), U8(s, MAV1CU_BUF_CDEFBUF),
                                               (long long)s->g.frame_bytes, U8(s, MAV1CU_BUF_LFMASK), num_cdef_presets);
    if (after_launch(s, "cdef")) return s->err;
  }
  return MAV1CU_OK;
}

extern "C" int mav1cu_cdef_select(mav1cu_session *s, int num_cdef_presets) {
  if (need_params(s)) return s->err;
  if (num_cdef_presets < 1 || num_cdef_presets > s->max_presets)
    return set_error(s, MAV1CU_ERR_ARG, "cdef_select: %d presets (session holds %d)", num_cdef_presets, s->max_presets);
  export_fence(s);
  flt::k_cdef_select<<<s->g.num_sbs, 256, 0, s->stream>>>(DP(s), U8(s, MAV1CU_BUF_SRC), U8(s, MAV1CU_BUF_CDEFBUF),
                                                           (long long)s->g.frame_bytes, U8(s, MAV1CU_BUF_REC),
                                                           (int8_t *)s->buf[MAV1CU_BUF_CDEF_CHOICE], num_cdef_presets);
  return after_launch(s, "cdef select");
}

extern "C" int mav1cu_restore(mav1cu_session *s) {
  if (need_params(s)) return s->err;
  int n = 3 * ((s->fp.frame_h + 3) >> 2) * ((s->fp.frame_w + 3) >> 2);
  flt::k_lr_apply<<<(n + 127) / 128, 128, 0, s->stream>>>(DP(s), U8(s, MAV1CU_BUF_REC), U8(s, MAV1CU_BUF_DBK),
                                                           U8(s, MAV1CU_BUF_LROUT),
                                                           (const LrUnit *)s->buf[MAV1CU_BUF_LRUNITS]);
  return after_launch(s, "loop restoration");
}

// Units of every plane of the current frame (the LRUNITS records in use).
static int lr_units_of(const FrameParams &fp) { return fp.lr_unit_off[2] + fp.lr_unit_rows[2] * fp.lr_unit_cols[2]; }

extern "C" int mav1cu_lr_search(mav1cu_session *s, int lr_test) {
  if (need_params(s)) return s->err;
  int n = lr_units_of(s->fp);
  if (n <= 0 || n > s->max_lr_units) return set_error(s, MAV1CU_ERR_ARG, "loop-restoration search: %d units", n);
  export_fence(s);  // LRUNITS and the plane types are exported
  s->lr_searched = 1;
  lrs::k_lr_fit<<<n, lrs::THREADS, sizeof(lrs::Shared), s->stream>>>(DP(s), U8(s, MAV1CU_BUF_REC),
                                                                       U8(s, MAV1CU_BUF_DBK), U8(s, MAV1CU_BUF_SRC),
                                                                       s->lrfit);
  if (after_launch(s, "loop-restoration fit")) return s->err;
  // the refinement's candidates under guessed references, for all units at
  // once: the serial choice below finds most of its SSEs cached
  lrs::k_lr_spec<<<n, lrs::THREADS, sizeof(lrs::Shared), s->stream>>>(DP(s), U8(s, MAV1CU_BUF_REC),
                                                                        U8(s, MAV1CU_BUF_DBK), U8(s, MAV1CU_BUF_SRC),
                                                                        s->lrfit);
  if (after_launch(s, "loop-restoration speculative refinement")) return s->err;
  lrs::k_lr_select<<<3, lrs::THREADS, sizeof(lrs::Shared), s->stream>>>(
      (FrameParams *)s->buf[MAV1CU_BUF_PARAMS], U8(s, MAV1CU_BUF_REC), U8(s, MAV1CU_BUF_DBK), U8(s, MAV1CU_BUF_SRC),
      s->lrfit, (LrUnit *)s->buf[MAV1CU_BUF_LRUNITS], lr_test, s->lr_types);
  return after_launch(s, "loop-restoration selection");
}

// ---- compact export of the writer inputs ------------------------------------------

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Section offsets of the export image; they depend on the geometry only.
static xport::Header export_layout(const mav1cu_session *s) {
  size_t nsb = (size_t)s->g.num_sbs;
  xport::Header h = {};
  h.num_sbs = (int32_t)nsb;
  h.sbs_off = 256;
  h.cdef_off = (int64_t)align256(h.sbs_off + nsb * sizeof(SbInfo));
  h.blocks_off = (int64_t)align256(h.cdef_off + nsb);
  h.coefs_off = (int64_t)align256(h.blocks_off + nsb * MAX_BLOCKS_PER_SB * sizeof(BlockInfo));
  h.params_off = (int64_t)align256(h.coefs_off + sizeof(int32_t) * COEFS_PER_SB * nsb);
  h.lr_off = (int64_t)align256(h.params_off + sizeof(FrameParams));
  h.rec_off = (int64_t)align256(h.lr_off + sizeof(LrUnit) * (size_t)s->max_lr_units);
  return h;
}

// Bytes of the visible I420 picture (mav1_get_recon's planes).
static size_t i420_bytes(const Geometry &g) {
  return (size_t)g.w * g.h + 2 * (size_t)((g.w + 1) >> 1) * ((g.h + 1) >> 1);
}

extern "C" size_t mav1cu_export_capacity(const mav1cu_session *s) {
  return (size_t)export_layout(s).rec_off + i420_bytes(s->g);
}

extern "C" void *mav1cu_export_image(mav1cu_session *s) {
  if (s->err) return NULL;
  if (!s->ximage && check_cuda(s, cudaHostAlloc(&s->ximage, mav1cu_export_capacity(s), cudaHostAllocMapped),
                               "export image allocation")) {
    s->ximage = NULL;
    return NULL;
  }
  return s->ximage;
}

extern "C" int mav1cu_export(mav1cu_session *s, void *image, size_t cap, int flags) {
  if (need_params(s)) return s->err;
  if (flags & ~(MAV1CU_EXPORT_REC | MAV1CU_EXPORT_LR))
    return set_error(s, MAV1CU_ERR_ARG, "export: unknown flags 0x%x", flags);
  size_t need = mav1cu_export_capacity(s);
  if (!image || cap < need || ((uintptr_t)image & 15))
    return set_error(s, MAV1CU_ERR_ARG, "export: image %p of %zu bytes (needs %zu bytes, 16-byte aligned)", image, cap,
                     need);
  cudaPointerAttributes a;
  if (check_cuda(s, cudaPointerGetAttributes(&a, image), "export: image attributes")) return s->err;
  uint8_t *dimg = NULL;
  int dev = 0;
  if (check_cuda(s, cudaGetDevice(&dev), "export: device")) return s->err;
  if (a.type == cudaMemoryTypeHost) dimg = (uint8_t *)a.devicePointer;
  else if ((a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == dev) dimg = (uint8_t *)image;
  if (!dimg)
    return set_error(s, MAV1CU_ERR_ARG,
                     "export: image %p is neither mapped page-locked host memory nor memory of device %d", image, dev);
  xport::Header layout = export_layout(s);
  layout.seq = ++s->xseq;
  int withRec = flags & MAV1CU_EXPORT_REC;
  layout.rec_bytes = withRec ? (int64_t)i420_bytes(s->g) : 0;
  layout.lr_units = (flags & MAV1CU_EXPORT_LR) && s->lr_searched ? lr_units_of(s->fp) : 0;
  if (layout.lr_units < 0 || layout.lr_units > s->max_lr_units)
    return set_error(s, MAV1CU_ERR_ARG, "export: %d loop-restoration units", layout.lr_units);
  size_t nsb = (size_t)s->g.num_sbs;
  const BlockInfo *blocks = (const BlockInfo *)s->buf[MAV1CU_BUF_BLOCKS];
  const SbInfo *sbs = (const SbInfo *)s->buf[MAV1CU_BUF_SBS];
  xport::Frame f = {s->fp.mi_cols, s->fp.mi_rows, s->fp.lossless};
  // fork: the transfer stream runs after the session's work so far
  if (check_cuda(s, cudaEventRecord(s->x_fork, s->stream), "export fork") ||
      check_cuda(s, cudaStreamWaitEvent(s->xs, s->x_fork, 0), "export fork"))
    return s->err;
  xport::k_export_count<<<(unsigned)((nsb + 7) / 8), 256, 0, s->xs>>>(f, blocks, sbs, (int)nsb, s->xcounts);
  if (after_launch(s, "export count")) return s->err;
  xport::k_export_scan<<<1, xport::SCAN_THREADS, 0, s->xs>>>(
      s->xcounts, (int)nsb, s->xblk_base, s->xcoef_base, s->xmeta, (const int8_t *)s->buf[MAV1CU_BUF_CDEF_CHOICE],
      dimg, layout, (long long)nsb * MAX_BLOCKS_PER_SB, (long long)nsb * COEFS_PER_SB);
  if (after_launch(s, "export scan")) return s->err;
  xport::k_export_write<<<(unsigned)imin((int)nsb, xport::STORE_CTAS), xport::WRITE_THREADS, 0, s->xs>>>(
      f, blocks, sbs, (int)nsb, (const int32_t *)s->buf[MAV1CU_BUF_COEFS], s->xblk_base, s->xcoef_base, s->xmeta,
      dimg, layout);
  if (after_launch(s, "export write")) return s->err;
  xport::k_export_side<<<1, 128, 0, s->xs>>>(s->fp, s->lr_types, (const LrUnit *)s->buf[MAV1CU_BUF_LRUNITS], dimg,
                                             layout);
  if (after_launch(s, "export parameters")) return s->err;
  if (withRec) {
    const Geometry &g = s->g;
    int rows = g.h + 2 * ((g.h + 1) >> 1);
    xport::k_export_rec<<<imin(rows, xport::STORE_CTAS), 128, 0, s->xs>>>(
        U8(s, MAV1CU_BUF_REC), make_int3(g.offset[0], g.offset[1], g.offset[2]),
                                                 make_int2(g.stride[0], g.stride[1]), g.w, g.h, s->xmeta,
                                                 dimg + layout.rec_off);
    if (after_launch(s, "export reconstruction")) return s->err;
  }
  if (check_cuda(s, cudaEventRecord(s->x_done, s->xs), "export done") ||
      check_cuda(s, cudaEventRecord(s->xring[layout.seq % XRING], s->xs), "export done"))
    return s->err;
  s->x_pending = 1;
  return MAV1CU_OK;
}

extern "C" void *mav1cu_host_alloc(size_t bytes) {
  void *p = NULL;
  if (cudaHostAlloc(&p, bytes ? bytes : 1, cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess) return NULL;
  return p;
}

extern "C" void mav1cu_host_free(void *p) {
  if (p) cudaFreeHost(p);
}

extern "C" int64_t mav1cu_export_seq(const mav1cu_session *s) { return s->xseq; }

// The device status word of the session (non-zero: a kernel gave up), read
// on the session's status stream: a copy into pageable host memory returns
// once it is done, and that stream orders after nothing else.
static int device_status(mav1cu_session *s) {
  int st = 0;
  if (cudaMemcpyAsync(&st, s->status, sizeof st, cudaMemcpyDeviceToHost, s->ss) != cudaSuccess ||
      cudaStreamSynchronize(s->ss) != cudaSuccess)
    return MAV1CU_ERR_CUDA;
  return st ? MAV1CU_ERR_DEVICE : MAV1CU_OK;
}

extern "C" int mav1cu_export_wait(mav1cu_session *s, int64_t seq) {
  if (seq <= 0 || seq > s->xseq) return MAV1CU_ERR_ARG;
  if (cudaSetDevice(s->device) != cudaSuccess) return MAV1CU_ERR_CUDA;
  if (cudaEventSynchronize(s->xring[seq % XRING]) != cudaSuccess) return MAV1CU_ERR_CUDA;
  return device_status(s);
}

extern "C" int mav1cu_export_query(mav1cu_session *s, int64_t seq) {
  if (seq <= 0 || seq > s->xseq) return MAV1CU_ERR_ARG;
  if (cudaSetDevice(s->device) != cudaSuccess) return MAV1CU_ERR_CUDA;
  cudaError_t e = cudaEventQuery(s->xring[seq % XRING]);
  if (e == cudaErrorNotReady) return 0;
  if (e != cudaSuccess) return MAV1CU_ERR_CUDA;
  int st = device_status(s);
  return st ? st : 1;
}


extern "C" int mav1cu_synchronize(mav1cu_session *s) {
  if (s->err) return s->err;
  if (check_cuda(s, cudaStreamSynchronize(s->stream), "synchronize")) return s->err;
  if (check_cuda(s, cudaStreamSynchronize(s->xs), "synchronize transfers")) return s->err;
  int st[2] = {0, 0};
  if (check_cuda(s, cudaMemcpy(st, s->status, sizeof st, cudaMemcpyDeviceToHost), "status")) return s->err;
  if (st[0])
    return set_error(s, MAV1CU_ERR_DEVICE, "device status %d: %s", st[0],
                     st[0] == 2   ? "a recon successor list overflowed"
                     : st[0] == 3 ? "a recon chroma-edge dependency wait gave up"
                     : st[0] == 4 ? "a recon source bulk-copy wait gave up"
                                  : "a recon ready-queue wait gave up");
  return MAV1CU_OK;
}

extern "C" const char *mav1cu_error_string(const mav1cu_session *s) { return s->err ? s->msg : ""; }
extern "C" int64_t mav1cu_launch_count(const mav1cu_session *s) { return s->launches; }

// ---- frame planning and the device-resident stream ------------------------------------

extern "C" int mav1cu_plan(const mav1cu_config *cfg, int nframes, mav1cu_frame_job *jobs, int cap) {
  if (!cfg || nframes < 0 || (nframes && !jobs)) return MAV1CU_ERR_ARG;
  drv::Planner pl;
  pl.n = drv::normalise(cfg);
  if (pl.n.c.altref > 0) pl.drain(nframes);
  else pl.low_delay(nframes);
  int n = (int)pl.jobs.size();
  if (n > cap) return MAV1CU_ERR_ARG;
  for (int i = 0; i < n; i++) jobs[i] = pl.jobs[i];
  return n;
}

extern "C" int mav1cu_plan_frames(const mav1cu_config *cfg, mav1cu_planner *state, int new_frames, int flush,
                                  mav1cu_frame_job *jobs, int cap) {
  if (!cfg || !state || new_frames < 0 || (cap > 0 && !jobs)) return MAV1CU_ERR_ARG;
  drv::Planner pl;
  pl.n = drv::normalise(cfg);
  pl.load(*state);
  if (pl.n.c.altref > 0) {
    pl.in_disp += new_frames;
    pl.inq_n += new_frames;
    pl.alt_drain(flush != 0);
  } else {
    for (int f = 0; f < new_frames; f++) pl.low_delay_frame();
  }
  int n = (int)pl.jobs.size();
  if (n > cap) return MAV1CU_ERR_ARG;  // the state is left unchanged
  for (int i = 0; i < n; i++) jobs[i] = pl.jobs[i];
  pl.store(state);
  return n;
}

extern "C" int mav1cu_layout_of(const mav1cu_config *cfg, mav1cu_layout *out) {
  if (!cfg || !out) return MAV1CU_ERR_ARG;
  drv::Norm n = drv::normalise(cfg);
  memset(out, 0, sizeof *out);
  out->cfg = n.c;
  out->leafopt_cfg = n.leafopt_cfg;
  out->mi_cols = n.mi_cols;
  out->mi_rows = n.mi_rows;
  out->sb_cols = n.sb_cols;
  out->sb_rows = n.sb_rows;
  out->num_sbs = n.sb_cols * n.sb_rows;
  out->tile_cols_log2 = n.tile_cols_log2;
  out->tile_cols = n.tile_cols;
  out->tile_w_sb = n.tile_w_sb;
  out->min_log2_tile_cols = n.min_log2_tile_cols;
  out->max_log2_tile_cols = n.max_log2_tile_cols;
  Geometry g = make_geometry(n.c.width, n.c.height);
  for (int p = 0; p < 3; p++) {
    out->stride[p] = g.stride[p];
    out->offset[p] = g.offset[p];
    out->plane_h[p] = g.plane_h[p];
  }
  out->frame_bytes = (int64_t)g.frame_bytes;
  return MAV1CU_OK;
}

extern "C" int mav1cu_frame_params_for(const mav1cu_config *cfg, const mav1cu_frame_job *job, mav1cu_frame_params *fp,
                                       int *num_cdef_presets) {
  if (!cfg || !job || !fp) return MAV1CU_ERR_ARG;
  drv::Norm n = drv::normalise(cfg);
  int presets = 0;
  drv::frame_params(n, *job, fp, &presets);
  if (num_cdef_presets) *num_cdef_presets = presets;
  return MAV1CU_OK;
}

// Frame engines: reference-chain frames (they refresh a slot) run on engine
// 0, non-reference frames on engine 1, each with its own session and CUDA
// stream (the reference's frame engines, encoder.c:1036-1176, with the same
// chain / leaf split). Slot reads and writes are ordered by CUDA events: a
// frame's reference copies wait for the slot's last write, and a slot write
// waits for every earlier frame that copied the slot's previous picture.
#define NUM_ENGINES 2

struct Event {
  cudaEvent_t e;
  Event() { cudaEventCreateWithFlags(&e, cudaEventDisableTiming); }
  ~Event() { cudaEventDestroy(e); }
};
typedef std::shared_ptr<Event> EventRef;

struct mav1cu_stream {
  drv::Norm n;
  mav1cu_session *eng[NUM_ENGINES];
  // host sources: per engine, an upload stream and two staging buffers, so
  // a frame's host->device copy overlaps the engine's previous frame
  uint8_t *staging[NUM_ENGINES][2];
  cudaStream_t upload[NUM_ENGINES];
  cudaEvent_t up_done[NUM_ENGINES][2], load_done[NUM_ENGINES][2];
  int up_next[NUM_ENGINES];
  uint8_t *slot[8];
  int64_t device_bytes;               // slots and staging (the engines count their own)
  EventRef written[8];                // last write of each slot
  std::vector<EventRef> readers[8];   // reference copies of the slot's picture since then
  size_t i420_bytes;
  int last_engine;
  // Motion-search planes per reference picture (the quarter-pel and
  // decimated planes depend on the picture alone): the engines' own plane
  // buffers serve as PLANE_SETS entries, each tagged with the picture it
  // holds. A reference frame's planes are built once, on its engine, right
  // after its slots are written; later frames that reference the picture use
  // them. Hazards are events: a user waits for `built`, a rebuild waits for
  // every motion search that read the entry's previous picture.
  struct PlaneSet {
    uint8_t *qp, *dref;
    int64_t pic = -1;               // picture held (-1: none)
    int64_t used = 0;               // last use, for least-recently-used replacement
    EventRef built;
    std::vector<EventRef> readers;
  } planes[2 * NUM_ENGINES];
  int64_t slot_pic[8];              // picture in each reference slot (-1: none)
  int64_t pic_seq, plane_clock;
};

// Entry holding picture `pic`, or -1.
static int plane_find(mav1cu_stream *st, int64_t pic) {
  for (int i = 0; i < 2 * NUM_ENGINES; i++)
    if (pic >= 0 && st->planes[i].pic == pic) return i;
  return -1;
}

// Builds the planes of picture `pic` (its samples in `ref`, padded layout)
// into the least recently used entry other than `keep`, on engine s's
// stream, after every reader of that entry's previous picture.
static int plane_build(mav1cu_stream *st, mav1cu_session *s, const uint8_t *ref, int64_t pic, int keep) {
  int v = -1;
  for (int i = 0; i < 2 * NUM_ENGINES; i++)
    if (i != keep && (v < 0 || st->planes[i].used < st->planes[v].used)) v = i;
  auto &e = st->planes[v];
  for (auto &r : e.readers) cudaStreamWaitEvent(s->stream, r->e, 0);
  e.readers.clear();
  if (build_ref_planes(s, ref, e.qp, e.dref)) return -1;
  e.built = std::make_shared<Event>();
  cudaEventRecord(e.built->e, s->stream);
  e.pic = pic;
  e.used = ++st->plane_clock;
  return v;
}

extern "C" int mav1cu_stream_create(const mav1cu_config *cfg, mav1cu_stream **out, char *err, size_t errlen) {
  *out = NULL;
  drv::Norm n = drv::normalise(cfg);
  mav1cu_stream *st = new mav1cu_stream();
  st->n = n;
  for (int e = 0; e < NUM_ENGINES; e++) {
    int rc = mav1cu_session_create(n.c.width, n.c.height, 4, &st->eng[e], err, errlen);
    if (rc) {
      mav1cu_stream_destroy(st);
      return rc;
    }
  }
  size_t fb = st->eng[0]->g.frame_bytes;
  st->i420_bytes = (size_t)n.c.width * n.c.height + 2 * (size_t)((n.c.width + 1) >> 1) * ((n.c.height + 1) >> 1);
  for (int i = 0; i < 2 * NUM_ENGINES; i++) {
    st->planes[i].qp = st->eng[i >> 1]->qp[i & 1];
    st->planes[i].dref = st->eng[i >> 1]->dref[i & 1];
  }
  for (int k = 0; k < 8; k++) st->slot_pic[k] = -1;
  cudaError_t e = cudaSuccess;
  for (int k = 0; k < 8 && e == cudaSuccess; k++) {
    e = cudaMalloc(&st->slot[k], fb);
    if (e == cudaSuccess) st->device_bytes += (int64_t)fb;
    if (e == cudaSuccess) e = cudaMemset(st->slot[k], 0, fb);
  }
  for (int k = 0; k < NUM_ENGINES && e == cudaSuccess; k++) {
    for (int b = 0; b < 2 && e == cudaSuccess; b++) {
      e = cudaMalloc(&st->staging[k][b], st->i420_bytes);
      if (e == cudaSuccess) st->device_bytes += (int64_t)st->i420_bytes;
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&st->up_done[k][b], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&st->load_done[k][b], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st->upload[k], cudaStreamNonBlocking);
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    snprintf(err, errlen, "stream allocation failed: %s", cudaGetErrorString(e));
    mav1cu_stream_destroy(st);
    return MAV1CU_ERR_NOMEM;
  }
  *out = st;
  return MAV1CU_OK;
}

extern "C" void mav1cu_stream_destroy(mav1cu_stream *st) {
  if (!st) return;
  for (int e = 0; e < NUM_ENGINES; e++) {
    if (st->upload[e]) cudaStreamSynchronize(st->upload[e]);
    if (st->eng[e]) cudaStreamSynchronize(st->eng[e]->stream);
  }
  for (int k = 0; k < 8; k++) {
    st->written[k].reset();
    st->readers[k].clear();
    if (st->slot[k]) cudaFree(st->slot[k]);
  }
  for (auto &p : st->planes) {
    p.built.reset();
    p.readers.clear();
  }
  for (int e = 0; e < NUM_ENGINES; e++) {
    for (int b = 0; b < 2; b++) {
      if (st->staging[e][b]) cudaFree(st->staging[e][b]);
      if (st->up_done[e][b]) cudaEventDestroy(st->up_done[e][b]);
      if (st->load_done[e][b]) cudaEventDestroy(st->load_done[e][b]);
    }
    if (st->upload[e]) cudaStreamDestroy(st->upload[e]);
    mav1cu_session_destroy(st->eng[e]);
  }
  delete st;
}

extern "C" mav1cu_session *mav1cu_stream_session(mav1cu_stream *st) { return st->eng[st->last_engine]; }

extern "C" int mav1cu_stream_reconfigure(mav1cu_stream *st, const mav1cu_config *cfg) {
  if (!cfg || cfg->width != st->n.c.width || cfg->height != st->n.c.height) return MAV1CU_ERR_ARG;
  int rc = mav1cu_stream_synchronize(st);
  if (rc) return rc;
  st->n = drv::normalise(cfg);
  for (int k = 0; k < 8; k++) {
    st->written[k].reset();
    st->readers[k].clear();
    st->slot_pic[k] = -1;
  }
  for (auto &p : st->planes) {
    p.pic = -1;
    p.built.reset();
    p.readers.clear();
  }
  return MAV1CU_OK;
}

extern "C" int64_t mav1cu_stream_device_bytes(const mav1cu_stream *st) {
  int64_t b = st->device_bytes;
  for (int k = 0; k < NUM_ENGINES; k++) b += st->eng[k]->device_bytes;
  return b;
}

extern "C" int64_t mav1cu_stream_bytes_for(const mav1cu_config *cfg) {
  if (!cfg || cfg->width < 16 || cfg->height < 16 || cfg->width > 65536 || cfg->height > 65536) return -1;
  Geometry g = make_geometry(cfg->width, cfg->height);
  int64_t i420 = (int64_t)cfg->width * cfg->height + 2 * (int64_t)((cfg->width + 1) >> 1) * ((cfg->height + 1) >> 1);
  return NUM_ENGINES * session_bytes(g, 4) + 8 * (int64_t)g.frame_bytes + NUM_ENGINES * 2 * i420;
}
extern "C" mav1cu_session *mav1cu_stream_engine(mav1cu_stream *st, int k) {
  return k >= 0 && k < NUM_ENGINES ? st->eng[k] : NULL;
}
extern "C" int mav1cu_stream_engines(const mav1cu_stream *st) { return NUM_ENGINES; }
extern "C" void *mav1cu_stream_slot(mav1cu_stream *st, int k) { return k >= 0 && k < 8 ? st->slot[k] : NULL; }

// Orders work: every engine waits for `stream`'s work so far (wait) / `stream`
// waits for every engine's work so far (join).
extern "C" int mav1cu_stream_wait(mav1cu_stream *st, void *stream) {
  Event ev;
  cudaEventRecord(ev.e, (cudaStream_t)stream);
  for (int k = 0; k < NUM_ENGINES; k++) {
    cudaStreamWaitEvent(st->eng[k]->stream, ev.e, 0);
    cudaStreamWaitEvent(st->upload[k], ev.e, 0);
  }
  return check_cuda(st->eng[0], cudaGetLastError(), "stream wait");
}

// The session's work so far, transfers included, precedes what `stream`
// enqueues next.
static void join_session(mav1cu_session *s, cudaStream_t stream) {
  Event ev, evx;
  cudaEventRecord(ev.e, s->stream);
  cudaStreamWaitEvent(stream, ev.e, 0);
  cudaEventRecord(evx.e, s->xs);
  cudaStreamWaitEvent(stream, evx.e, 0);
}

extern "C" int mav1cu_stream_join(mav1cu_stream *st, void *stream) {
  for (int k = 0; k < NUM_ENGINES; k++) join_session(st->eng[k], (cudaStream_t)stream);
  return check_cuda(st->eng[0], cudaGetLastError(), "stream join");
}
extern "C" int mav1cu_stream_synchronize(mav1cu_stream *st) {
  for (int k = 0; k < NUM_ENGINES; k++) {
    if (check_cuda(st->eng[k], cudaStreamSynchronize(st->upload[k]), "synchronize uploads")) return st->eng[k]->err;
    if (mav1cu_synchronize(st->eng[k])) return st->eng[k]->err;
  }
  return MAV1CU_OK;
}

// Slots the reference encoder keeps (encoder.c:129-136): ALTREF driver 0, 2, 3
// (and 4..7 with pyramid leaf frames); low-delay path LAST 0 and GOLDEN 1.
static int slot_exists(const drv::Norm &n, int k) {
  if (n.c.altref) return k == 0 || k == 2 || k == 3 || (n.c.leaf && k >= 4);
  return k == 0 || (k == 1 && n.c.multi_ref);
}

extern "C" int mav1cu_stream_encode(mav1cu_stream *st, const mav1cu_frame_job *job, const void *i420, int on_device) {
  const mav1cu_config &c = st->n.c;
  int rf = job->is_key ? 0xFF : job->refresh;
  int ei = rf ? 0 : 1;  // reference chain on engine 0, leaf frames on engine 1
  mav1cu_session *s = st->eng[ei];
  if (s->err) return s->err;
  st->last_engine = ei;
  size_t fb = s->g.frame_bytes;
  const uint8_t *src = (const uint8_t *)i420;
  int b = -1;
  if (!on_device) {
    // upload stream: wait until the load that last read this staging buffer
    // is done, copy, and let the engine wait for the copy
    b = st->up_next[ei];
    st->up_next[ei] ^= 1;
    cudaStream_t us = st->upload[ei];
    if (check_cuda(s, cudaStreamWaitEvent(us, st->load_done[ei][b], 0), "source upload") ||
        check_cuda(s, cudaMemcpyAsync(st->staging[ei][b], i420, st->i420_bytes, cudaMemcpyHostToDevice, us),
                   "source upload") ||
        check_cuda(s, cudaEventRecord(st->up_done[ei][b], us), "source upload") ||
        check_cuda(s, cudaStreamWaitEvent(s->stream, st->up_done[ei][b], 0), "source upload"))
      return s->err;
    src = st->staging[ei][b];
  }
  dim3 grid((s->g.stride[0] + 511) / 512, (s->g.plane_h[0] + drv::LS_ROWS - 1) / drv::LS_ROWS, 3);
  drv::k_load_source<<<grid, dim3(32, drv::LS_ROWS), 0, s->stream>>>(src, U8(s, MAV1CU_BUF_SRC), c.width, c.height,
                                                                    s->g.sb_cols, s->g.sb_rows);
  if (after_launch(s, "load source")) return s->err;
  if (b >= 0 && check_cuda(s, cudaEventRecord(st->load_done[ei][b], s->stream), "source upload")) return s->err;
  if (!job->is_key) {
    int refs[2] = {job->last_slot, job->arf_slot};
    int bufs[2] = {MAV1CU_BUF_REF, MAV1CU_BUF_GOLD};
    for (int r = 0; r < 2; r++) {
      int k = refs[r];
      if (k < 0) continue;
      if (k > 7) return set_error(s, MAV1CU_ERR_ARG, "stream: bad reference slot %d", k);
      if (st->written[k]) cudaStreamWaitEvent(s->stream, st->written[k]->e, 0);
      if (check_cuda(s, cudaMemcpyAsync(s->buf[bufs[r]], st->slot[k], fb, cudaMemcpyDeviceToDevice, s->stream), "reference copy"))
        return s->err;
    }
    EventRef in = std::make_shared<Event>();
    cudaEventRecord(in->e, s->stream);
    for (int r = 0; r < 2; r++)
      if (refs[r] >= 0) st->readers[refs[r]].push_back(in);
  }
  FrameParams fp;
  int presets = 0;
  drv::frame_params(st->n, *job, &fp, &presets);
  if (mav1cu_set_params(s, &fp)) return s->err;
  // the motion search's reference planes from the per-picture cache: a hit
  // waits for the build, a miss builds them here from this frame's copy
  int mePlanes = !fp.frame_is_intra && (fp.turbo & T_ME_HPEL), used[2] = {-1, -1};
  if (mePlanes) {
    int nref = fp.golden ? 2 : 1, refs[2] = {job->last_slot, job->arf_slot};
    int64_t pic[2];
    for (int r = 0; r < nref; r++) {
      pic[r] = refs[r] >= 0 ? st->slot_pic[refs[r]] : -1;
      used[r] = plane_find(st, pic[r]);
    }
    for (int r = 0; r < nref; r++) {
      if (used[r] < 0) used[r] = plane_find(st, pic[r]);  // the other reference may have built it
      if (used[r] >= 0) {
        cudaStreamWaitEvent(s->stream, st->planes[used[r]].built->e, 0);
        st->planes[used[r]].used = ++st->plane_clock;
      } else {
        // not cached (replaced, or a slot never written): a picture of its own
        if (pic[r] < 0) pic[r] = ++st->pic_seq;
        used[r] = plane_build(st, s, U8(s, r ? MAV1CU_BUF_GOLD : MAV1CU_BUF_REF), pic[r], used[1 - r]);
        if (used[r] < 0) return s->err;
      }
      s->ext_qp[r] = st->planes[used[r]].qp;
      s->ext_dref[r] = st->planes[used[r]].dref;
    }
  }
  if (!fp.frame_is_intra && mav1cu_motion_search(s)) return s->err;
  if (mePlanes) {
    EventRef rd = std::make_shared<Event>();
    cudaEventRecord(rd->e, s->stream);
    for (int r = 0; r < 2; r++)
      if (used[r] >= 0 && (r == 0 || used[1] != used[0])) st->planes[used[r]].readers.push_back(rd);
  }
  if (frame_core_after_me(s)) return s->err;
  // filter stage gating of run_frame_core (encoder.c:617-632)
  int nPresets = c.cdef ? 4 : 0, cdefOff = (job->leafopt & 4) != 0;
  int lfOn = fp.lf_level[0] || fp.lf_level[1] || fp.lf_level[2] || fp.lf_level[3];
  int filt = lfOn || (nPresets && !cdefOff) || !c.turbo;
  if (filt && (mav1cu_filter_info(s) || mav1cu_filter(s, presets))) return s->err;
  // loop restoration (encoder.c:633-643): the deblocked frame is kept before
  // CDEF selection, the search runs on the CDEF output, the restored frame
  // replaces REC
  int useLr = c.restoration && c.qindex > 0 && !(job->leafopt & 8);
  if (useLr && mav1cu_copy(s, MAV1CU_BUF_DBK, MAV1CU_BUF_REC, fb)) return s->err;
  if (c.cdef && c.qindex > 0 && !cdefOff && mav1cu_cdef_select(s, nPresets)) return s->err;
  if (useLr && (mav1cu_lr_search(s, c.lr_test) || mav1cu_copy(s, MAV1CU_BUF_LROUT, MAV1CU_BUF_REC, fb) ||
                mav1cu_restore(s) || mav1cu_copy(s, MAV1CU_BUF_REC, MAV1CU_BUF_LROUT, fb)))
    return s->err;
  EventRef out;
  for (int k = 0; k < 8; k++) {
    if (!((rf >> k) & 1) || !slot_exists(st->n, k)) continue;
    for (auto &r : st->readers[k]) cudaStreamWaitEvent(s->stream, r->e, 0);
    if (st->written[k]) cudaStreamWaitEvent(s->stream, st->written[k]->e, 0);
    if (check_cuda(s, cudaMemcpyAsync(st->slot[k], s->buf[MAV1CU_BUF_REC], fb, cudaMemcpyDeviceToDevice, s->stream), "slot"))
      return s->err;
  }
  if (rf) {
    out = std::make_shared<Event>();
    cudaEventRecord(out->e, s->stream);
    int64_t pic = ++st->pic_seq;
    int any = 0;
    for (int k = 0; k < 8; k++)
      if (((rf >> k) & 1) && slot_exists(st->n, k)) {
        st->written[k] = out;
        st->readers[k].clear();
        st->slot_pic[k] = pic;
        any = 1;
      }
    // a new reference picture: its motion-search planes, once, from REC
    // (the slots' copy source), for every later frame that references it
    if (any && (fp.turbo & T_ME_HPEL) && plane_build(st, s, U8(s, MAV1CU_BUF_REC), pic, -1) < 0) return s->err;
  }
  return check_cuda(s, cudaGetLastError(), "stream encode");
}

// ---- the counting build (-DMAV1CU_COUNT, libmav1cu_count.so) ----------------------
#ifdef MAV1CU_COUNT
#include "mav1cu_count.h"

extern "C" int mav1cu_work_read(uint64_t *out, int n) {
  if (!out || n < W_COUNT) return MAV1CU_ERR_ARG;
  unsigned long long v[W_COUNT];
  if (cudaDeviceSynchronize() != cudaSuccess || cudaMemcpyFromSymbol(v, d_work, sizeof v) != cudaSuccess)
    return MAV1CU_ERR_CUDA;
  for (int i = 0; i < W_COUNT; i++) out[i] = v[i];
  return W_COUNT;
}

extern "C" int mav1cu_work_reset(void) {
  unsigned long long z[W_COUNT] = {};
  if (cudaDeviceSynchronize() != cudaSuccess || cudaMemcpyToSymbol(d_work, z, sizeof z) != cudaSuccess)
    return MAV1CU_ERR_CUDA;
  return cudaDeviceSynchronize() == cudaSuccess ? MAV1CU_OK : MAV1CU_ERR_CUDA;
}

namespace {
// Independent 32-bit integer chains per thread: per element and iteration a
// multiply-add (the FMA pipe) and an exclusive-or plus an add (the ALU
// pipe), 4 operations, none of which the compiler can merge.
constexpr int PEAK_CHAINS = 8;
__global__ void __launch_bounds__(256) k_int_peak(unsigned *out, int iters, unsigned seed) {
  unsigned a[PEAK_CHAINS], b[PEAK_CHAINS];
  for (int k = 0; k < PEAK_CHAINS; k++) {
    a[k] = threadIdx.x * (k + 1) + seed;
    b[k] = blockIdx.x ^ (seed * (k + 7));
  }
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int k = 0; k < PEAK_CHAINS; k++) {
      a[k] = a[k] * 2654435761u + b[k];
      b[k] = (b[k] ^ a[k]) + 0x9e3779b9u;
    }
  }
  unsigned s = 0;
  for (int k = 0; k < PEAK_CHAINS; k++) s += a[k] ^ b[k];
  if (s == seed) out[0] = s;  // keeps the chains live; practically never true
}
}  // namespace

extern "C" int mav1cu_work_int_peak(double *ops_per_s) {
  if (!ops_per_s) return MAV1CU_ERR_ARG;
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  unsigned *out = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaMalloc(&out, sizeof(unsigned)) != cudaSuccess) return MAV1CU_ERR_NOMEM;
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int iters = 4096, ctas = sms * 8, threads = 256;
  float best = 0;
  for (int r = 0; r < 4; r++) {
    cudaEventRecord(e0, st);
    k_int_peak<<<ctas, threads, 0, st>>>(out, iters, 12345u + r);
    cudaEventRecord(e1, st);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (r > 0 && (best == 0 || ms < best)) best = ms;
  }
  cudaError_t e = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  cudaFree(out);
  if (e != cudaSuccess || best <= 0) return MAV1CU_ERR_CUDA;
  *ops_per_s = 4.0 * PEAK_CHAINS * (double)iters * ctas * threads / (best * 1e-3);
  return MAV1CU_OK;
}
#endif
