/* ORACLE — test infrastructure only; never linked into the product.
 *
 * The reference's tile writer (src/tile_writer.c) compiled in place from the
 * reference checkout. Its single libdispatch call (tile_writer.c:610,
 * dispatch_apply over the tile columns with a clang Blocks literal) cannot be
 * parsed by gcc, so the macro below swallows that one statement, the
 * reference's write_tile is renamed out of the way, and write_tile
 * (tile_writer.c:603-627) is restated after the include with a plain loop
 * over the tile columns (tiles code disjoint columns of e->mi, so the order
 * does not change any byte). */
#define dispatch_apply(...) ((void)0)
#define write_tile oracle_write_tile_reference_unused
#include "tile_writer.c"
#undef write_tile

/* tile_writer.c:603-627: code every tile column; all but the last tile are
 * preceded by tile_size_minus_1 as le(4). */
size_t write_tile(struct Mav1Encoder *e, uint8_t **out) {
  memset(e->mi, 0, sizeof(MiInfo) * e->mi_rows * e->mi_cols);
  for (int i = 0; i < e->num_sbs; i++) e->cdef_idx[i] = -1;
  mvpred_frame_start(e);
  int n = e->tile_cols;
  uint8_t **bufs = calloc((size_t)n, sizeof *bufs);
  size_t *sizes = calloc((size_t)n, sizeof *sizes);
  for (int tc = 0; tc < n; tc++) sizes[tc] = write_one_tile(e, tc, &bufs[tc]);
  size_t total = 0;
  for (int i = 0; i < n; i++) total += sizes[i] + (i < n - 1 ? 4 : 0);
  uint8_t *o = malloc(total ? total : 1), *q = o;
  for (int i = 0; i < n; i++) {
    if (i < n - 1) {
      uint32_t m1 = (uint32_t)sizes[i] - 1;
      for (int b = 0; b < 4; b++) *q++ = (uint8_t)(m1 >> (8 * b));
    }
    memcpy(q, bufs[i], sizes[i]);
    q += sizes[i];
    free(bufs[i]);
  }
  free(bufs);
  free(sizes);
  *out = o;
  return total;
}
