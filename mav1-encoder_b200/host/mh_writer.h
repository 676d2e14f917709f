/* Interface between the Linux host driver (encoder_cuda.c) and the glue over
 * the reference's entropy coder and OBU writer (writer.c).
 *
 * writer.c is the only translation unit that sees the reference encoder's
 * internal state (src/enc_internal.h): it keeps one "writer view" of that
 * state per context, filled from a frame description, so the reference's
 * tile writer (src/tile_writer.c), MV prediction (src/mvpred.c) and OBU
 * writer (src/obu.c) run unchanged on the writer inputs the device exported.
 * Nothing here depends on the reference's headers. */
#ifndef MH_WRITER_H
#define MH_WRITER_H

#include <stddef.h>
#include <stdint.h>

#include "mav1cu.h"

typedef struct mh_writer mh_writer;

/* One coded frame as the writer needs it. */
typedef struct {
  const mav1cu_frame_job *job;
  const mav1cu_frame_params *fp;  /* setup_params' record (host copy) */
  int low_delay;                  /* mav1_encode's path (no ALTREF driver) */
  int last_hint, arf_hint;        /* OrderHint of the LAST / second reference slot (-1: none) */
  int ref_hint[7];                /* OrderHint of the slot of each ref_frame_idx (ALTREF driver) */
  /* writer inputs: the sections of the export image */
  const mav1cu_sb_info *sbs;
  const mav1cu_block_info *blocks;
  const int32_t *coefs;
  const int8_t *cdef_choice;
  const mav1cu_lr_unit *lrunits;  /* NULL: no loop restoration */
} mh_frame;

/* A writer context for frames of this layout (MiInfo grid, CDEF indices and
 * the writer view); NULL on allocation failure. */
mh_writer *mh_writer_new(const mav1cu_layout *layout);
void mh_writer_free(mh_writer *w);
/* Takes a new configuration of the same frame size (a restarted encoder). */
void mh_writer_config(mh_writer *w, const mav1cu_layout *layout);
/* Points the context at a frame: fills the frame header (FrameHdr) the way
 * the reference driver does (alt_code, encoder.c:1004-1030; mav1_encode,
 * encoder.c:822-846; setup_params' header fields, encoder.c:467-509). */
void mh_writer_frame(mh_writer *w, const mh_frame *f);
/* write_tile's set-up (tile_writer.c:603-606): the tile columns can then be
 * coded concurrently (they touch disjoint columns of the MiInfo grid). */
void mh_writer_begin(mh_writer *w);
/* Codes tile column tc (write_one_tile, tile_writer.c:553-598); *out is
 * malloc'ed. */
size_t mh_writer_tile(mh_writer *w, int tc, uint8_t **out);
int mh_writer_tile_cols(const mh_writer *w);
/* OBUs of the frame: the frame OBU over the assembled tile data
 * (write_frame_obu, obu.c:217) and, for key frames, the sequence header. */
size_t mh_writer_frame_obu(mh_writer *w, const uint8_t *tile, size_t tileSize, uint8_t *out);
size_t mh_writer_sequence_header(mh_writer *w, uint8_t *out);
/* The frame's MAV1_DUMP_DEC record (encoder.c:659-704), malloc'ed, *bytes
 * long; the driver appends the records to the file in coding order. */
uint8_t *mh_writer_dump_record(mh_writer *w, size_t tileSize, size_t *bytes);
/* Block statistics of the frame (frame_tail's count, encoder.c:711-720;
 * count_tools, encoder.c:565-579): num_blocks, num_inter_blocks, tool_use[16]. */
void mh_writer_stats(mh_writer *w, int *numBlocks, int *numInter, int toolUse[16]);

size_t mh_temporal_delimiter(uint8_t *out);
size_t mh_show_existing(int slot, uint8_t *out);

#endif
