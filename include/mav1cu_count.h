/* mav1cu_count.h - the counting build of the backend (libmav1cu_count.so).
 *
 * No counterpart in the reference: this is measurement support. The same
 * kernels as libmav1cu.so, compiled with -DMAV1CU_COUNT, add the algorithmic
 * work units they perform to device counters (one per category below);
 * every entry point of mav1cu.h is present and behaves the same. The
 * product library has none of this.
 */
#ifndef MAV1CU_COUNT_H
#define MAV1CU_COUNT_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Categories, in counter order (units in parentheses):
 *  0 motion search full-pel SAD, full resolution (byte pairs)
 *  1 motion search full-pel SAD, 4x4-decimated planes (byte pairs)
 *  2 motion search sub-pel 4x4 SATD (units)
 *  3 quarter-pel planes (filter taps: horizontal pass over the window, vertical per output)
 *  4 analysis 4x4 SATD (units)
 *  5 analysis inter prediction (samples, 8-tap horizontal + vertical each)
 *  6 analysis intra prediction (samples)
 *  7 analysis CfL alpha search ((sample, alpha) SSE terms)
 *  8 reconstruction inter prediction (samples, 8-tap horizontal + vertical each)
 *  9 reconstruction intra prediction (samples)
 * 10 forward transform (multiply-accumulates of both matrix passes)
 * 11 quantiser (coefficients)
 * 12 inverse transform (operations: 3 log2 N per point of each N-point 1D pass)
 * 13 deblocking (filter taps: the filter length of every filtered sample line)
 * 14 CDEF (taps: 8 projections per sample of the direction search, 12 per filtered sample)
 * 15 loop restoration (taps per restored sample: 14 Wiener, 34 self-guided) */
#define MAV1CU_WORK_COUNT 16

/* Copies the counters (since the last reset) into out[0 .. n - 1] after a
 * device synchronisation. Returns the number of counters, or an error code
 * (n < MAV1CU_WORK_COUNT: -1). */
int mav1cu_work_read(uint64_t *out, int n);
/* Zeroes the counters (synchronises the device first). */
int mav1cu_work_reset(void);
/* Measured peak rate of 32-bit integer operations of the current device:
 * independent multiply-add, exclusive-or and add chains on every SM (a
 * multiply-add counts as two operations), best of three timed launches. */
int mav1cu_work_int_peak(double *ops_per_s);

#ifdef __cplusplus
}
#endif

#endif
