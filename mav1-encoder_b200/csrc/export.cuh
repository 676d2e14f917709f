// Compact export of a frame's entropy-coder inputs: the superblock table,
// the blocks in use and the quantised levels of the coded planes, packed on
// the device into one image that the caller's host memory receives directly
// (page-locked, mapped memory: the kernels' stores cross PCIe / C2C, so the
// amount copied need not be known when the work is enqueued).
//
// The reference's host steps reach blocks only through sbs[s].first_block
// (tile_writer.c:585, encoder.c:327,337,519,678,717) and levels only through
// coef_off[plane] + txIdx * tw * th (tile_writer.c:437-456), so an image
// with both rewritten is read by them unchanged:
//  - blocks: each superblock's num_blocks records, back to back in
//    superblock order; first_block is the running count;
//  - levels: for every block that is not skipped (some eob[] != 0), every
//    plane with eob[plane] != 0 gets the levels its in-frame transform blocks
//    hold, up to the last one the writer reads (plane_levels), back to back
//    in block order; its coef_off points there.
//    Every plane with eob[plane] == 0 of such a block reads zeros: its
//    coef_off is 0, and the image's level section opens with a run of zeros
//    as long as the largest such plane. Skipped blocks read no levels
//    (tile_writer.c:429-436) and keep coef_off 0.
// Level count <= the dense buffer's: the zero run is no longer than the
// plane it replaces, which is not copied.
#pragma once

#include <stddef.h>

#include "common.cuh"

namespace xport {

constexpr int SB_WORDS = (int)(sizeof(SbInfo) / 4);
constexpr int BLK_WORDS = (int)(sizeof(BlockInfo) / 4);
constexpr int WRITE_THREADS = 128;
constexpr int SCAN_THREADS = 1024;
// CTAs of the kernels that store into the image: the stores are paced by the
// bus, and a small persistent grid leaves the other SMs (and their shared
// memory) to the frame engines the export overlaps
#ifndef MAV1CU_STORE_CTAS
#define MAV1CU_STORE_CTAS 16
#endif
constexpr int STORE_CTAS = MAV1CU_STORE_CTAS;

struct Header {  // mav1cu_export_header
  int32_t status, seq, num_sbs, num_blocks, num_coefs, zero_run;
  int64_t sbs_off, cdef_off, blocks_off, coefs_off, rec_off, rec_bytes, bytes;
  int64_t params_off, lr_off;
  int32_t lr_units, pad;
};
static_assert(sizeof(Header) == 104, "export header layout");

// The frame parameters (the host's record, passed by value, with lr_type as
// the loop-restoration search chose it) and the LR units in use, into their
// sections. The rest of the image is written by the other export kernels.
__global__ void k_export_side(FrameParams fp, const int *lrTypes, const LrUnit *units, uint8_t *image, Header layout) {
  int *pdst = (int *)(image + layout.params_off);
  const int *psrc = (const int *)&fp;
  const int nparams = (int)(sizeof(FrameParams) / 4), lrType = (int)(offsetof(FrameParams, lr_type) / 4);
  int t = blockIdx.x * blockDim.x + threadIdx.x, n = gridDim.x * blockDim.x;
  for (int k = t; k < nparams; k += n)
    pdst[k] = layout.lr_units > 0 && k >= lrType && k < lrType + 3 ? lrTypes[k - lrType] : psrc[k];
  int *udst = (int *)(image + layout.lr_off);
  const int *usrc = (const int *)units;
  int nwords = layout.lr_units * (int)(sizeof(LrUnit) / 4);
  for (int k = t; k < nwords; k += n) udst[k] = usrc[k];
}

// The frame parameters the packing depends on, passed by value: the export
// runs on its own stream and must not read PARAMS, which the next frame's
// set-up rewrites.
struct Frame {
  int mi_cols, mi_rows, lossless;
};

// Levels of `plane` of block b that the writer may read: the plane's
// transform blocks whose start lies inside the frame, tw * th apart
// (tile_writer.c:437-456, transform size as tile_writer.c:360,439); the
// writer reads a transform block's levels only at its scan positions
// (find_eob, k_recon.h:50-54; write_coeffs, tile_writer.c:177-178,228-229),
// which lie inside the adjusted transform (at most 32 x 32, the first
// min(32, tw) * min(32, th) levels), so the run ends there.
HD int plane_levels(const Frame &f, const BlockInfo &b, int plane) {
  int bs = b.bsize, sub = plane > 0;
  int txSz = f.lossless ? TX_4X4
             : plane == 0 ? (b.is_inter ? T(Max_Tx_Size_Rect)[bs] : depth_tx_size(bs, b.tx_depth))
                          : uv_tx_size(bs, 1, 1);
  int tw = T(Tx_Width)[txSz], th = T(Tx_Height)[txSz];
  int psz = T(Subsampled_Size)[bs][sub][sub];
  int pw = block_w(psz), ph = block_h(psz);
  int maxX = (f.mi_cols * 4) >> sub, maxY = (f.mi_rows * 4) >> sub;
  int x0 = (b.mi_col >> sub) * 4, y0 = (b.mi_row >> sub) * 4;
  int nx = imin((pw + tw - 1) / tw, (imax(0, maxX - x0) + tw - 1) / tw);
  int ny = imin((ph + th - 1) / th, (imax(0, maxY - y0) + th - 1) / th);
  int ntx = nx * ny;
  return ntx ? (ntx - 1) * tw * th + imin(32, tw) * imin(32, th) : 0;
}

HD int block_skipped(const BlockInfo &b) { return b.eob[0] == 0 && b.eob[1] == 0 && b.eob[2] == 0; }

// Per superblock: blocks, copied levels, longest zero-level plane, and 1 in
// .w when its table entry or blocks point outside the session's buffers (the
// write kernel reads only ranges checked here). One warp per superblock,
// lanes over its blocks.
__global__ void k_export_count(Frame f, const BlockInfo *blocks, const SbInfo *sbs, int num_sbs, int4 *counts) {
  int sb = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (sb >= num_sbs) return;
  long long nblk = (long long)num_sbs * MAX_BLOCKS_PER_SB, ncoef = (long long)num_sbs * COEFS_PER_SB;
  int nb = sbs[sb].num_blocks, first = sbs[sb].first_block;
  int bad = nb < 0 || nb > MAX_BLOCKS_PER_SB || first < 0 || (long long)first + nb > nblk;
  if (bad) nb = 0;
  int coded = 0, zmax = 0;
  for (int k = lane; k < nb; k += 32) {
    const BlockInfo &b = blocks[first + k];
    if (block_skipped(b)) continue;
    if (b.bsize < 0 || b.bsize > BLOCK_64X16 || b.tx_depth < 0 || b.tx_depth > 4) {
      bad = 1;
      continue;
    }
    for (int p = 0; p < 3; p++) {
      int n = plane_levels(f, b, p);
      if (b.eob[p]) {
        coded += n;
        bad |= b.coef_off[p] < 0 || (b.coef_off[p] & 3) || (long long)b.coef_off[p] + n > ncoef;
      } else {
        zmax = imax(zmax, n);
      }
    }
  }
  for (int o = 16; o; o >>= 1) {
    coded += __shfl_xor_sync(0xffffffffu, coded, o);
    zmax = imax(zmax, __shfl_xor_sync(0xffffffffu, zmax, o));
    bad |= __shfl_xor_sync(0xffffffffu, bad, o);
  }
  if (lane == 0) counts[sb] = make_int4(nb, coded, zmax, bad);
}

// Exclusive scans of the block and level counts, the zero run, the header,
// the zero run's levels and the CDEF choices. One CTA. meta[0] receives the
// zero run, meta[1] 1 when the blocks are valid and the image fits its
// capacity; otherwise nothing but the header is written and its status is
// 2 (invalid blocks) or 1 (over capacity).
__global__ void __launch_bounds__(SCAN_THREADS) k_export_scan(const int4 *counts, int num_sbs, int *blk_base,
                                                                int *coef_base, int *meta, const int8_t *cdef,
                                                                uint8_t *image, Header layout, long long cap_blocks,
                                                                long long cap_coefs) {
  __shared__ int wsum[2][SCAN_THREADS / 32];
  __shared__ int wmax[SCAN_THREADS / 32];
  __shared__ int carry[2], zrun, invalid;
  int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) carry[0] = carry[1] = 0;
  int zmax = 0, bad = 0;
  __syncthreads();
  for (int base = 0; base < num_sbs; base += SCAN_THREADS) {
    int i = base + tid;
    int4 v = i < num_sbs ? counts[i] : make_int4(0, 0, 0, 0);
    zmax = imax(zmax, v.z);
    bad |= v.w;
    int a = v.x, c = v.y;
    for (int o = 1; o < 32; o <<= 1) {
      int ta = __shfl_up_sync(0xffffffffu, a, o), tc = __shfl_up_sync(0xffffffffu, c, o);
      if (lane >= o) {
        a += ta;
        c += tc;
      }
    }
    if (lane == 31) {
      wsum[0][warp] = a;
      wsum[1][warp] = c;
    }
    __syncthreads();
    if (warp == 0) {
      int sa = wsum[0][lane], sc = wsum[1][lane];
      for (int o = 1; o < 32; o <<= 1) {
        int ta = __shfl_up_sync(0xffffffffu, sa, o), tc = __shfl_up_sync(0xffffffffu, sc, o);
        if (lane >= o) {
          sa += ta;
          sc += tc;
        }
      }
      wsum[0][lane] = sa;
      wsum[1][lane] = sc;
    }
    __syncthreads();
    int pa = carry[0] + (warp ? wsum[0][warp - 1] : 0) + a - v.x;
    int pc = carry[1] + (warp ? wsum[1][warp - 1] : 0) + c - v.y;
    if (i < num_sbs) {
      blk_base[i] = pa;
      coef_base[i] = pc;
    }
    __syncthreads();
    if (tid == 0) {
      carry[0] += wsum[0][SCAN_THREADS / 32 - 1];
      carry[1] += wsum[1][SCAN_THREADS / 32 - 1];
    }
    __syncthreads();
  }
  for (int o = 16; o; o >>= 1) {
    zmax = imax(zmax, __shfl_xor_sync(0xffffffffu, zmax, o));
    bad |= __shfl_xor_sync(0xffffffffu, bad, o);
  }
  if (lane == 0) wmax[warp] = zmax | (bad ? 1 << 30 : 0);
  __syncthreads();
  if (tid == 0) {
    int z = 0, anyBad = 0;
    for (int w = 0; w < SCAN_THREADS / 32; w++) {
      z = imax(z, wmax[w] & ((1 << 30) - 1));
      anyBad |= wmax[w] >> 30;
    }
    zrun = z;
    invalid = anyBad;
  }
  __syncthreads();
  long long nblocks = carry[0], ncoefs = (long long)zrun + carry[1];
  int fits = !invalid && nblocks <= cap_blocks && ncoefs <= cap_coefs;
  if (tid == 0) {
    meta[0] = zrun;
    meta[1] = fits;
  }
  if (fits) {
    int4 *z4 = (int4 *)(image + layout.coefs_off);
    for (int k = tid; k < zrun / 4; k += SCAN_THREADS) z4[k] = make_int4(0, 0, 0, 0);
    int8_t *cd = (int8_t *)(image + layout.cdef_off);
    for (int k = tid; k < num_sbs; k += SCAN_THREADS) cd[k] = cdef[k];
  }
  if (tid == 0) {
    Header h = layout;
    h.status = invalid ? 2 : fits ? 0 : 1;
    h.num_blocks = (int32_t)nblocks;
    h.num_coefs = (int32_t)ncoefs;
    h.zero_run = zrun;
    h.bytes = fits ? (long long)sizeof(Header) + (long long)num_sbs * (SB_WORDS * 4 + 1) + nblocks * BLK_WORDS * 4 +
                         ncoefs * 4 + (long long)sizeof(FrameParams) + (long long)layout.lr_units * sizeof(LrUnit) +
                         layout.rec_bytes
                   : (long long)sizeof(Header);
    if (!fits) h.rec_bytes = 0;
    *(Header *)image = h;
  }
}

// One superblock: its table entry, its blocks with coef_off rewritten, and
// the levels of its coded planes. Shared state: the CTA's.
__device__ void write_sb(const Frame &f, const BlockInfo *blocks, const SbInfo *sbs, int sb, const int32_t *coefs,
                         const int *blk_base, const int *coef_base, const int *meta, uint8_t *image,
                         const Header &layout, BlockInfo *sblk, int *rel4, int *src4, int *wtot) {
  int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const SbInfo &s = sbs[sb];
  int nb = imin(s.num_blocks, MAX_BLOCKS_PER_SB), first = s.first_block, bb = blk_base[sb];
  int zrun = meta[0], cbase = zrun + coef_base[sb];
  const int32_t *sw = (const int32_t *)&s;
  int32_t *dsb = (int32_t *)(image + layout.sbs_off) + (size_t)sb * SB_WORDS;
  for (int w = tid; w < SB_WORDS; w += WRITE_THREADS) dsb[w] = w == 0 ? bb : sw[w];
  const int32_t *bw = (const int32_t *)(blocks + first);
  for (int w = tid; w < nb * BLK_WORDS; w += WRITE_THREADS) ((int32_t *)sblk)[w] = bw[w];
  __syncthreads();
  // levels of each block (thread k <-> block k), then a scan over the blocks
  int n[3] = {0, 0, 0};
  if (tid < nb && !block_skipped(sblk[tid]))
    for (int p = 0; p < 3; p++)
      if (sblk[tid].eob[p]) n[p] = plane_levels(f, sblk[tid], p);
  int tot = n[0] + n[1] + n[2], x = tot;
  for (int o = 1; o < 32; o <<= 1) {
    int t = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += t;
  }
  if (lane == 31) wtot[warp] = x;
  __syncthreads();
  int pre = x - tot;
  for (int w = 0; w < warp; w++) pre += wtot[w];
  int total = 0;
  for (int w = 0; w < WRITE_THREADS / 32; w++) total += wtot[w];
  if (tid < nb) {
    BlockInfo &b = sblk[tid];
    int off = pre;
    for (int p = 0; p < 3; p++) {
      rel4[tid * 3 + p] = off >> 2;
      src4[tid * 3 + p] = b.coef_off[p] >> 2;
      b.coef_off[p] = n[p] ? cbase + off : 0;
      off += n[p];
    }
  }
  __syncthreads();
  int32_t *dblk = (int32_t *)(image + layout.blocks_off) + (size_t)bb * BLK_WORDS;
  for (int w = tid; w < nb * BLK_WORDS; w += WRITE_THREADS) dblk[w] = ((const int32_t *)sblk)[w];
  // levels: int4 index i of this superblock's run belongs to the last item
  // whose start is <= i (empty items share their successor's start)
  int items = 3 * nb, total4 = total >> 2;
  const int4 *c4 = (const int4 *)coefs;
  int4 *d4 = (int4 *)(image + layout.coefs_off) + (cbase >> 2);
  for (int i = tid; i < total4; i += WRITE_THREADS) {
    int lo = 0, hi = items - 1;
    while (lo < hi) {
      int mid = (lo + hi + 1) >> 1;
      if (rel4[mid] <= i) lo = mid;
      else hi = mid - 1;
    }
    d4[i] = __ldcs(c4 + src4[lo] + (i - rel4[lo]));
  }
}

// STORE_CTAS CTAs, striding over the superblocks.
__global__ void __launch_bounds__(WRITE_THREADS) k_export_write(Frame f, const BlockInfo *blocks, const SbInfo *sbs,
                                                                 int num_sbs, const int32_t *coefs,
                                                                 const int *blk_base, const int *coef_base,
                                                                 const int *meta, uint8_t *image, Header layout) {
  __shared__ BlockInfo sblk[MAX_BLOCKS_PER_SB];
  __shared__ int rel4[3 * MAX_BLOCKS_PER_SB], src4[3 * MAX_BLOCKS_PER_SB];
  __shared__ int wtot[WRITE_THREADS / 32];
  if (!meta[1]) return;
  for (int sb = blockIdx.x; sb < num_sbs; sb += gridDim.x) {
    write_sb(f, blocks, sbs, sb, coefs, blk_base, coef_base, meta, image, layout, sblk, rel4, src4, wtot);
    __syncthreads();  // this superblock's shared state is consumed
  }
}

// The shown reconstruction as mav1_get_recon returns it (encoder.c:877-915):
// the visible w x h luma samples, then the (w+1)/2 x (h+1)/2 samples of each
// chroma plane, rows packed. STORE_CTAS CTAs stride over the output rows;
// 16-byte stores where the row width and both row starts allow.
__global__ void k_export_rec(const uint8_t *rec, int3 offset, int2 stride, int w, int h, const int *meta,
                             uint8_t *dst) {
  if (!meta[1]) return;
  int cw = (w + 1) >> 1, ch = (h + 1) >> 1;
  for (int row = blockIdx.x; row < h + 2 * ch; row += gridDim.x) {
    int p = row < h ? 0 : row < h + ch ? 1 : 2;
    int r = p == 0 ? row : p == 1 ? row - h : row - h - ch;
    int pw = p ? cw : w;
    const uint8_t *s = rec + (p == 0 ? offset.x : p == 1 ? offset.y : offset.z) + (size_t)r * (p ? stride.y : stride.x);
    uint8_t *d = dst + (p == 0 ? (size_t)r * w : (size_t)w * h + (size_t)(p - 1) * cw * ch + (size_t)r * cw);
    if (!(pw & 15) && !((uintptr_t)s & 15) && !((uintptr_t)d & 15)) {
      for (int k = threadIdx.x; k < pw / 16; k += blockDim.x) ((int4 *)d)[k] = __ldcs((const int4 *)s + k);
    } else {
      for (int k = threadIdx.x; k < pw; k += blockDim.x) d[k] = s[k];
    }
  }
}

}  // namespace xport
