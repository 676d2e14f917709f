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

#ifdef __cplusplus
}
#endif

#endif
