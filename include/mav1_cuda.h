/*
 * libmav1.so — the mav1 encoder API (src/mav1.h of neolite/mav1-encoder,
 * unchanged: mav1_create, mav1_send_frame, mav1_receive_packet,
 * mav1_get_recon, ...) on the B200 encode backend, plus the extensions
 * below. A caller of the reference links this library instead of the
 * reference's libmav1.a; tools/mav1enc.c builds against it unchanged.
 *
 * Behaviour differences from the reference library:
 *  - every frame is coded on the GPU (libmav1cu.so); a configuration with
 *    use_metal = 0 (the CPU backend, --cpu) is refused by mav1_create;
 *  - packets come out as their frames complete, like the reference's
 *    concurrent (frame engine) mode; without ALTREF, mav1_send_frame returns
 *    once the frame's packet is ready, like mav1_encode;
 *  - environment: MAV1_CUDA_THREADS (host entropy threads of the process,
 *    default: the online CPUs), MAV1_CUDA_IMAGES (export images per frame
 *    engine, default 8: frames in flight between the device and the host
 *    entropy coder), and the reference's MAV1_* knobs of the frame driver.
 */
#ifndef MAV1_CUDA_H
#define MAV1_CUDA_H

#include <stdint.h>

#include "mav1.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Totals of an encoder since mav1_create. No counterpart in the reference
 * (its buffers are shared with the GPU through unified memory, so nothing
 * crosses a bus). */
typedef struct {
  int64_t frames;        /* coded frames (hidden ALTREF frames included) */
  int64_t h2d_bytes;     /* source bytes copied host -> device */
  int64_t d2h_bytes;     /* export image bytes written device -> host (writer inputs and reconstructions) */
  double entropy_s;      /* host thread time in entropy coding and OBU writing */
} mav1_cuda_counters;

void mav1_cuda_get_counters(const Mav1Encoder *e, mav1_cuda_counters *out);

/* Device memory an encoder holds (its frame engines, reference slots and
 * staging: requested bytes), and what mav1_create would allocate for a
 * configuration; -1 for an unsupported one. For admission of encoders
 * against a device-memory budget. */
int64_t mav1_cuda_device_bytes(const Mav1Encoder *e);
int64_t mav1_cuda_device_bytes_for(const Mav1Config *cfg);

/* Starts a new clip on an existing encoder, keeping its device memory and
 * host buffers: waits until every frame sent so far is coded, drops packets
 * not yet received, and takes cfg (same width and height; the rest may
 * change). The next frame sent starts the new clip with a key frame; the
 * bitstream equals a fresh encoder's. For servers that reuse encoders across
 * sessions (creating and destroying device memory synchronises the GPU for
 * every other encoder). Returns 0, or -1 for another frame size. */
int mav1_cuda_restart(Mav1Encoder *e, const Mav1Config *cfg);

#ifdef __cplusplus
}
#endif

#endif
