// mav1cu_edge_types_noalloc: the intra edge filter types of every block,
// the same result as mav1cu_edge_types, for callers that may not allocate
// device memory.
//
// Who needs it: a host that carves all of a GPU's memory into fixed pools
// when it starts (a serving process with a hard HBM budget, several encoder
// engines sharing one device) and must not see an allocation fail later;
// and a host whose other streams are busy, where cudaMalloc / cudaFree can
// synchronise the device and stall them. The session API allocates its
// scratch at session creation; this entry point takes the caller's device
// buffers as they are and keeps its own scratch in a fixed device array.
//
// Scratch: two byte maps of mi_rows * mi_cols cells (the "smooth" mark of
// each 4x4 unit for luma, then for chroma) in the static array below, at
// most MAX_MI cells each (frames up to 4096 x 4096 luma samples; 2 MiB in
// all). Each call zeroes the 2 * mi_rows * mi_cols bytes it uses on the
// caller's stream before it writes them, so nothing depends on what a
// previous call left there. There is one array per device and per process:
// calls that overlap in time on one device (on different streams, or from
// different host threads) share it and race; order such calls on one stream
// or with events.
//
// Set-up: every call looks up the array's device address with
// cudaGetSymbolAddress while the caller's device is current (the address is
// not cached: after cudaDeviceReset, or once the primary context is
// destroyed and made again, the array may sit elsewhere). The first call on
// a device may load the library's device code on it: make that first call
// before any stream capture on the device.
//
// Sizes: mi_rows / mi_cols must equal the frame's (params->mi_rows /
// mi_cols); the scratch is sized by them. Blocks at or beyond that size are
// left unchanged, so a caller passing a smaller size than the frame's gets
// those blocks' bits 4 / 5 as they were.
//
// The algorithm is get_filter_type( ) of the AV1 specification (7.11.2) as
// the reference runs it on the host (src/encoder.c:319-346): mark every 4x4
// unit covered by a block that is intra with a SMOOTH* mode, then set each
// block's bit 4 (luma) / bit 5 (chroma) of interp_filter when the above or
// left neighbour unit is marked.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>

#include "common.cuh"

namespace noalloc {

constexpr int MAX_MI = 1024 * 1024;  // 4x4 units per map: 4096 x 4096 luma

static __device__ __align__(256) uint8_t scratch[2 * MAX_MI];

HD int smooth(int m) { return m == SMOOTH_PRED || m == SMOOTH_V_PRED || m == SMOOTH_H_PRED; }

// One CTA per superblock, one thread per block of it (at most
// MAX_BLOCKS_PER_SB). rows / cols are the caller's frame size in 4x4 units;
// block positions outside it are skipped, so no write leaves the maps.
__global__ void k_marks(const BlockInfo *blocks, const SbInfo *sbs, int rows, int cols, uint8_t *ys, uint8_t *uvs) {
  int k = threadIdx.x;
  const SbInfo &sb = sbs[blockIdx.x];
  if (k >= imin(sb.num_blocks, MAX_BLOCKS_PER_SB)) return;
  const BlockInfo *b = &blocks[sb.first_block + k];
  if (b->mi_row < 0 || b->mi_col < 0) return;
  int ysm = !b->is_inter && smooth(b->y_mode), uvsm = !b->is_inter && smooth(b->uv_mode);
  int r1 = imin(rows, b->mi_row + T(Num_4x4_Blocks_High)[b->bsize]);
  int c1 = imin(cols, b->mi_col + T(Num_4x4_Blocks_Wide)[b->bsize]);
  for (int r = b->mi_row; r < r1; r++)
    for (int c = b->mi_col; c < c1; c++) {
      ys[r * cols + c] = (uint8_t)ysm;
      uvs[r * cols + c] = (uint8_t)uvsm;
    }
}

__global__ void k_types(const FrameParams *fp, BlockInfo *blocks, const SbInfo *sbs, int rows, int cols,
                        const uint8_t *ys, const uint8_t *uvs) {
  int k = threadIdx.x;
  const SbInfo &sb = sbs[blockIdx.x];
  if (k >= imin(sb.num_blocks, MAX_BLOCKS_PER_SB)) return;
  BlockInfo *b = &blocks[sb.first_block + k];
  int r = b->mi_row, c = b->mi_col;
  if (r < 0 || c < 0 || r >= rows || c >= cols) return;
  int availU = r > 0, availL = c > tile_col_start(fp, c);
  int fy = (availU && ys[(r - 1) * cols + c]) || (availL && ys[r * cols + c - 1]);
  int fuv = (availU && uvs[(r - 1) * cols + imin(c + 1, cols - 1)]) || (availL && uvs[imin(r + 1, rows - 1) * cols + c - 1]);
  b->interp_filter = (b->interp_filter & 15) | fy << 4 | fuv << 5;
}

static int fail(char *err, size_t errlen, int rc, const char *fmt, ...) {
  if (err && errlen) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, errlen, fmt, ap);
    va_end(ap);
  }
  return rc;
}

}  // namespace noalloc

extern "C" int mav1cu_edge_types_noalloc(const mav1cu_frame_params *params, mav1cu_block_info *blocks,
                                         const mav1cu_sb_info *sbs, int mi_rows, int mi_cols, int num_sbs,
                                         void *stream, char *err, size_t errlen) {
  using namespace noalloc;
  if (!params || !blocks || !sbs)
    return fail(err, errlen, MAV1CU_ERR_ARG, "edge types (no-alloc): null device pointer");
  if (mi_rows <= 0 || mi_cols <= 0 || num_sbs <= 0)
    return fail(err, errlen, MAV1CU_ERR_ARG, "edge types (no-alloc): non-positive size %d x %d, %d superblocks",
                mi_rows, mi_cols, num_sbs);
  if ((long long)mi_rows * mi_cols > MAX_MI)
    return fail(err, errlen, MAV1CU_ERR_ARG,
                "edge types (no-alloc): %d x %d 4x4 units exceed the scratch limit of %d units "
                "(4096 x 4096 luma samples)",
                mi_rows, mi_cols, MAX_MI);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return fail(err, errlen, MAV1CU_ERR_CUDA, "edge types (no-alloc): cudaGetDevice: %s", cudaGetErrorString(e));
  void *p = nullptr;
  e = cudaGetSymbolAddress(&p, scratch);
  if (e != cudaSuccess || !p)
    return fail(err, errlen, MAV1CU_ERR_CUDA, "edge types (no-alloc): scratch address on device %d: %s", dev,
                cudaGetErrorString(e));
  uint8_t *base = (uint8_t *)p;
  size_t cells = (size_t)mi_rows * mi_cols;
  uint8_t *ys = base, *uvs = base + cells;
  cudaStream_t st = (cudaStream_t)stream;
  e = cudaMemsetAsync(base, 0, 2 * cells, st);
  if (e != cudaSuccess)
    return fail(err, errlen, MAV1CU_ERR_CUDA, "edge types (no-alloc): clearing scratch: %s", cudaGetErrorString(e));
  k_marks<<<num_sbs, MAX_BLOCKS_PER_SB, 0, st>>>(blocks, sbs, mi_rows, mi_cols, ys, uvs);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return fail(err, errlen, MAV1CU_ERR_CUDA, "edge types (no-alloc): marks launch: %s", cudaGetErrorString(e));
  k_types<<<num_sbs, MAX_BLOCKS_PER_SB, 0, st>>>(params, blocks, sbs, mi_rows, mi_cols, ys, uvs);
  e = cudaGetLastError();
  if (e != cudaSuccess)
    return fail(err, errlen, MAV1CU_ERR_CUDA, "edge types (no-alloc): types launch: %s", cudaGetErrorString(e));
  return MAV1CU_OK;
}
