/*
 * dpkem_wire.h: framed request/response records for KEM serving, and a shared-memory
 * ring through which another process feeds them to a frame server (libdpkem.so).
 *
 * No counterpart in the reference: its drivers run one fixed batch per program
 * (FrodoKEM976-GPU/main.cu:13-34, SABER-GPU/main.cu:12-38).  The payloads are the
 * reference's object layouts (FrodoKEM976-GPU/include/api.h:7-10,
 * SABER-GPU/include/params.h:27-48), in the argument order of dpkem_*_batch.
 *
 * Frame = 32-byte header + payload sections; all integers little-endian.  Each section
 * starts at a 16-byte multiple within the frame and a frame is a multiple of 32 bytes, so
 * a block of frames that starts 32-byte aligned keeps every section aligned as the
 * kernels need it.
 *
 *   request  keypair: header | coins                  (Frodo 64 B, Saber 96 B)
 *            encaps:  header | coins (pad 16) | pk     (Frodo 24 B coins, Saber 32 B)
 *            decaps:  header | ct | sk
 *   response keypair: header | pk | sk
 *            encaps:  header | ct | ss (pad 16)
 *            decaps:  header | ss (pad 16)
 * then zero padding up to the 32-byte multiple given in frame_bytes.  A response carries
 * the request's scheme, op and id; a decapsulation that fails the re-encryption check
 * still answers DPKEM_OK (implicit rejection).  A DPKEM_FRAME_PAD header marks filler
 * to be skipped (it closes the end of a ring).
 */
#ifndef DPKEM_WIRE_H
#define DPKEM_WIRE_H

#include <stddef.h>
#include <stdint.h>

#include "dpkem.h"

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define DPKEM_FRAME_MAGIC 0x464B5044u /* "DPKF" */
#define DPKEM_FRAME_PAD 0x504B5044u   /* "DPKP": filler, skip frame_bytes */
#define DPKEM_FRAME_VERSION 1u
#define DPKEM_FRAME_HEADER 32u
#define DPKEM_FRAME_ALIGN 32u

enum { DPKEM_OP_KEYPAIR = 0, DPKEM_OP_ENC = 1, DPKEM_OP_DEC = 2 };

typedef struct {
  uint32_t magic;       /* DPKEM_FRAME_MAGIC or DPKEM_FRAME_PAD */
  uint8_t version;      /* DPKEM_FRAME_VERSION */
  uint8_t scheme;       /* DPKEM_FRODO976 / DPKEM_LIGHTSABER / DPKEM_SABER / DPKEM_FIRESABER */
  uint8_t op;           /* DPKEM_OP_* */
  int8_t status;        /* responses: DPKEM_OK; requests: 0 */
  uint64_t id;          /* caller's request id, echoed in the response */
  uint32_t frame_bytes; /* whole frame including this header, a multiple of 32 */
  uint32_t reserved[3]; /* zero */
} dpkem_frame_header;

/* Byte sizes of the request and the response frame of (scheme, op). */
int dpkem_frame_bytes(int scheme, int op, size_t *request_bytes, size_t *response_bytes);

/* Host-only check of a block of request frames: counts them (PAD frames are skipped and
 * not counted) and sums the response bytes.  With max_frames > 0 it stops after that many
 * frames; *used_bytes is then the length of the prefix it took.  DPKEM_EINVAL on a bad
 * header (magic, version, scheme, op, or a frame_bytes other than the request size) or a
 * frame that runs past the block. */
int dpkem_frames_scan(const uint8_t *req, size_t req_bytes, size_t max_frames, size_t *n_frames,
                      size_t *used_bytes, size_t *response_bytes);

/* Runs every request frame of a host block on the GPU and writes the response frames,
 * in request order, into `resp` (capacity resp_cap; *resp_bytes = bytes written).
 * The block is copied to the device once per pipeline chunk, the payloads are read and
 * written in place by the persistent mixed-batch kernel, a small kernel writes the
 * response headers, and each chunk's responses are copied back once.  For full copy
 * bandwidth register both host ranges (dpkem_host_register) or use pinned memory.
 * Synchronous: returns when the responses are in `resp`. */
int dpkem_frames_run(dpkem_ctx *ctx, int form, const uint8_t *req, size_t req_bytes, uint8_t *resp,
                     size_t resp_cap, size_t *resp_bytes);

/* Page-lock a caller's host range (for example a shared-memory ring) for direct DMA. */
int dpkem_host_register(void *ptr, size_t bytes);
int dpkem_host_unregister(void *ptr);

/* ---- shared-memory ring -------------------------------------------------------------
 * One mapping holds a 4096-byte control page, then the request ring, then the response
 * ring, each `capacity` bytes (a multiple of 4096).  Counters are monotonic byte counts
 * (position = count % capacity), each on its own 64-byte line, published with release
 * stores and read with acquire loads.  A frame never straddles the end of a ring: a
 * writer that lacks the room before the end closes it with a PAD frame (as soon as the
 * PAD itself fits) and continues at 0, so every frame no larger than the ring gets
 * through once the reader catches up.
 * Producer (client): dpkem_ring_push, then dpkem_ring_pop for the responses.
 * Server: dpkem_ring_serve (loop), or dpkem_ring_acquire / dpkem_frames_run /
 * dpkem_ring_release by hand. */
#define DPKEM_RING_MAGIC 0x524B5044u /* "DPKR" */
#define DPKEM_RING_CONTROL 4096u

typedef struct {
  uint32_t magic, version;
  uint64_t capacity;
  uint8_t pad0[48];
  uint64_t req_tail;  /* written by the client */
  uint8_t pad1[56];
  uint64_t req_head;  /* written by the server */
  uint8_t pad2[56];
  uint64_t resp_tail; /* written by the server */
  uint8_t pad3[56];
  uint64_t resp_head; /* written by the client */
  uint8_t pad4[56];
  uint64_t stop;      /* nonzero: dpkem_ring_serve returns */
  uint8_t pad5[56];
  uint64_t served;    /* frames answered so far (server) */
} dpkem_ring_control;

/* Bytes of a ring mapping with `capacity` bytes per direction. */
size_t dpkem_ring_bytes(size_t capacity);
/* Initialise a zeroed mapping of dpkem_ring_bytes(capacity) bytes. */
int dpkem_ring_init(void *base, size_t capacity);
/* Client: append the longest prefix of whole request frames (validated) that fits;
 * *pushed = bytes of `frames` taken.  DPKEM_EAGAIN if not even one frame fits yet;
 * DPKEM_EINVAL for a frame larger than the ring. */
int dpkem_ring_push(void *base, const uint8_t *frames, size_t bytes, size_t *pushed);
/* Client: move whole response frames (PAD skipped) into out; *got = bytes copied (0 if
 * none), *n_frames (if non-null) = frames copied. */
int dpkem_ring_pop(void *base, uint8_t *out, size_t cap, size_t *got, size_t *n_frames);
/* Server, one batch at a time: take up to max_frames contiguous request frames and
 * reserve room for their responses (call dpkem_ring_release before the next acquire).  Offsets are relative to each ring's start; *req_advance / *resp_advance
 * include PAD bytes and are what dpkem_ring_release publishes.  DPKEM_EAGAIN: nothing
 * to take, or no room for even one response; DPKEM_EINVAL: a bad frame, or a response
 * larger than the ring. */
int dpkem_ring_acquire(void *base, size_t max_frames, size_t *req_off, size_t *req_bytes, size_t *req_advance,
                       size_t *resp_off, size_t *resp_bytes, size_t *resp_advance, size_t *n_frames);
int dpkem_ring_release(void *base, size_t req_advance, size_t resp_advance, size_t n_frames);
/* Server loop until control->stop is set: batches of up to max_frames request frames are
 * taken at the server's own cursors and run on ctxs[0..nctx) in turn, so up to nctx
 * batches are in flight (copies of one overlapping the kernels of another); responses
 * are published strictly in request order.  Sleeps idle_us microseconds when idle.
 * Register the mapping with dpkem_host_register first. */
int dpkem_ring_serve(dpkem_ctx *const *ctxs, int nctx, int form, void *base, size_t max_frames, int idle_us);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif /* DPKEM_WIRE_H */
