/*
 * dpkem: batched FrodoKEM-976-SHAKE and Saber (LightSaber / Saber / FireSaber) KEM
 * engine for NVIDIA B200 (sm_100a).  C ABI of libdpkem.so.
 *
 * Drop-in boundary for the reference (benlwk/DPCrypto) batched entry points:
 *   - frodoKEMKeypair / frodoKEMEncap / frodoKEMDecap replace
 *     FrodoKEM976-GPU/include/cuda_kernel.cuh:7-9 (batch = compile-time BLOCK there,
 *     dpkem_set_compat_batch() here);
 *   - saber_enc / saber_dec replace SABER-GPU/include/cuda_kernel.cuh:6-7
 *     (mode 0 = DP / dp4a form, 1 = INT32 schoolbook, as in the reference; 2 selects the
 *     int8 tensor-core form).
 *   - dpkem_{keypair,enc,dec}_batch are the batched form of the PQClean-style API the
 *     reference's headers declare (FrodoKEM976-GPU/include/api.h:14-18), with explicit
 *     coins so every call is reproducible.
 * Byte layouts are the reference's: arrays of n contiguous instances, stride = object size.
 *   Frodo-976: pk 15632 = seedA(16) || BE16(B); sk 31296 = s || pk || LE16(S^T) || H(pk);
 *              ct 15744 = BE16(B') || BE16(C); ss 24          (FrodoKEM976-GPU/include/api.h:7-10)
 *   Saber l:   pk 320l+32, sk 416l + pk + 64, ct 320l + eT*32, ss 32 (SABER-GPU/include/params.h:27-48)
 * Coins: Frodo keypair 64 B = s || seedSE || z, Frodo enc 24 B = mu;
 *        Saber keypair 96 B = seed_A || seed_s || z, Saber enc 32 B.
 */
#ifndef DPKEM_H
#define DPKEM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* Status codes (the reference returns void and checks no CUDA error). */
enum {
  DPKEM_OK = 0,
  DPKEM_EINVAL = -1,       /* bad scheme/form/size/pointer/alignment */
  DPKEM_ENOMEM = -2,       /* allocation failed or the request exceeds the HBM budget */
  DPKEM_ECUDA = -3,        /* a CUDA runtime call failed */
  DPKEM_ETIMEOUT = -4,     /* a bounded device wait expired (the kernel unwound) */
  DPKEM_EUNSUPPORTED = -5, /* valid request the library does not implement */
  DPKEM_EAGAIN = -6        /* non-blocking ring call: nothing to take / no room yet (dpkem_wire.h) */
};

/* Schemes: the value of a Saber scheme is its module rank l.  DPKEM_FRODO976AES is
 * FrodoKEM-976-AES: sizes, layouts and every step as DPKEM_FRODO976 except that A is
 * generated with AES-128 (A[i][j..j+7] = AES128(seedA, LE16(i) || LE16(j) || 0^12)); the
 * reference declares it (FrodoKEM976-GPU/include/aes.h, gen_a_mat_mul.cuh:6-7) but never
 * implements it. */
enum { DPKEM_FRODO976 = 0, DPKEM_FRODO976AES = 1, DPKEM_LIGHTSABER = 2, DPKEM_SABER = 3, DPKEM_FIRESABER = 4 };

/* Product forms. */
enum { DPKEM_FORM_DP4A = 0, DPKEM_FORM_INT32 = 1, DPKEM_FORM_TC = 2 };

/* Flags. */
#define DPKEM_FLAG_DEVICE_PTRS 1u /* all buffers are device pointers (pk/ct arrays 16-byte, others 8-byte aligned); call is async */

typedef struct dpkem_ctx dpkem_ctx;

/* Create a context on `device` whose scratch arena may use at most `hbm_budget_bytes`
 * (0 = default 8 GiB).  Batches larger than the budget allows run in chunks. */
int dpkem_ctx_create(dpkem_ctx **out, int device, size_t hbm_budget_bytes);
int dpkem_ctx_destroy(dpkem_ctx *ctx);
/* Cap the CTAs of this context's persistent launches (mixed batches, graphs, frames):
 * 0 (default) = two per SM, the whole GPU.  A server that runs several contexts at once
 * gives each a share, so a launch never queues behind another one's resident CTAs. */
int dpkem_ctx_set_max_ctas(dpkem_ctx *ctx, int max_ctas);

/* Grow the context's device arena to at least `bytes` now (within its HBM budget), so
 * that no later call has to: regrowing frees the old arena, which waits for the whole
 * device.  dpkem_mixed_bytes(scheme, n) is the arena a mixed batch of n requests of that
 * scheme needs (Frodo requests need the most); 0 for an unknown scheme. */
int dpkem_ctx_reserve(dpkem_ctx *ctx, size_t bytes);

/* Diagnostics for the failure path: runs a kernel whose bounded device wait cannot be
 * satisfied (which = 0: an mbarrier that no thread arrives on, the tensor stages' wait;
 * 1: a persistent-kernel task whose dependency never completes, the mixed batches' wait)
 * and returns what a real expiry returns, DPKEM_ETIMEOUT, after the 2 s limit.  Nothing
 * traps; the context stays usable. */
int dpkem_selftest_timeout(dpkem_ctx *ctx, int which);
size_t dpkem_mixed_bytes(int scheme, size_t n);

/* Object sizes in bytes; any pointer may be NULL. */
int dpkem_sizes(int scheme, size_t *pk, size_t *sk, size_t *ct, size_t *ss, size_t *kp_coins, size_t *enc_coins);

/* Largest batch one launch chain processes under the context's budget (host-pointer mode). */
size_t dpkem_max_chunk(dpkem_ctx *ctx, int scheme);

/* Batched operations.  `stream` is a cudaStream_t (NULL = the context's stream).
 * Host-pointer mode (flags 0): copies in, computes, copies out, returns when done.
 * Device-pointer mode: enqueues on `stream` and returns; call dpkem_sync() for the
 * device error word.  Decaps failure is not an error (implicit rejection). */
int dpkem_keypair_batch(dpkem_ctx *ctx, int scheme, int form, size_t n, const uint8_t *coins, uint8_t *pk,
                        uint8_t *sk, unsigned flags, void *stream);
int dpkem_enc_batch(dpkem_ctx *ctx, int scheme, int form, size_t n, const uint8_t *coins, const uint8_t *pk,
                    uint8_t *ct, uint8_t *ss, unsigned flags, void *stream);
int dpkem_dec_batch(dpkem_ctx *ctx, int scheme, int form, size_t n, const uint8_t *ct, const uint8_t *sk,
                    uint8_t *ss, unsigned flags, void *stream);

/* ---- Mixed batches: one persistent launch over mixed schemes and operations ----
 * Each request names a scheme, an operation and its device buffers (pk/ct 16-byte, others 8-byte aligned),
 * in the argument order of the batched calls:
 *   keypair: in0 = coins, out0 = pk, out1 = sk
 *   encaps:  in0 = coins, in1 = pk, out0 = ct, out1 = ss
 *   decaps:  in0 = ct,    in1 = sk, out0 = ss
 * The requests run as one launch of persistent CTAs that pull stage tasks from a device
 * work queue; results equal those of the batched calls on the same inputs.  No
 * counterpart in the reference (one scheme per compiled program, fixed launch chains). */
typedef struct {
  int32_t scheme; /* DPKEM_FRODO976 / DPKEM_FRODO976AES / DPKEM_LIGHTSABER / DPKEM_SABER / DPKEM_FIRESABER */
  int32_t op;     /* 0 keypair, 1 encaps, 2 decaps */
  const uint8_t *in0, *in1;
  uint8_t *out0, *out1;
} dpkem_request;

/* Enqueue on `stream` (NULL = context stream); dpkem_sync() reports device-side errors. */
int dpkem_mixed_batch(dpkem_ctx *ctx, int form, size_t n, const dpkem_request *reqs, void *stream);

/* The same, with device-drawn randomness: a keypair or encaps request whose in0 (coins) is
 * NULL gets coins = SHAKE256(key[0..32) || LE64(first + i) || "kp" / "enc"), i = its
 * position in reqs, truncated to the scheme's coin length, computed inside the persistent
 * kernel by the request's first stage (no host-to-device randomness).  With key = 00 01 ..
 * 1F these are the dpkem_coins streams. */
int dpkem_mixed_batch_keyed(dpkem_ctx *ctx, int form, size_t n, const dpkem_request *reqs, const uint8_t *key,
                            uint64_t first, void *stream);

/* The same batch captured once as a CUDA graph (its own device memory) and replayed. */
typedef struct dpkem_graph dpkem_graph;
int dpkem_mixed_graph_create(dpkem_ctx *ctx, int form, size_t n, const dpkem_request *reqs, dpkem_graph **out);
int dpkem_mixed_graph_launch(dpkem_graph *g, void *stream);
int dpkem_mixed_graph_destroy(dpkem_graph *g);

/* ---- KEM service: one long-lived launch that admits requests while it runs ----
 * Requests (dpkem_request, device buffers, the mixed batches' layout and alignment) are
 * appended to a ring the running kernel reads: the kernel's CTAs admit them into
 * per-(scheme, operation, stage) ready queues in device memory and pull stage work from
 * those queues (thread-level stages gather whatever instances are ready, across
 * submissions), so a request never waits for an earlier launch to drain.  Each accepted
 * request gets a ticket (consecutive from 0); the last stage writes it into host-mapped
 * memory and dpkem_service_poll() returns the tickets that have completed.  Results equal
 * the batched calls on the same inputs.  Input buffers must hold their data when submitted
 * and stay untouched, and outputs unread, until the request's ticket is returned.
 * Admission is live: a request is accepted while a ring slot is free and the scratch
 * records of the requests in flight leave room for its own (FrodoKEM 31,744 bytes, Saber
 * 2,816 / 4,864 / 7,936 bytes for l = 2 / 3 / 4); the rest of a submission is left to the caller
 * to resubmit.
 * The kernel ends after idle_ms without work and is relaunched by the next submit, poll or
 * drain.  Every device wait is bounded; an expired one makes poll / drain / close return
 * DPKEM_ETIMEOUT.  While a service is open its launch holds the CTA slots it was given
 * (dpkem_ctx_set_max_ctas caps them): other kernels on the device share what is left.
 * No counterpart in the reference (FrodoKEM976-GPU/main.cu:13-34, SABER-GPU/main.cu:12-38
 * run one fixed batch per program). */
typedef struct dpkem_service dpkem_service;
typedef struct {
  uint32_t max_inflight;   /* ring slots: requests submitted and not yet completed (rounded up to a power of 2) */
  uint32_t idle_ms;        /* the launch ends after this long without work (relaunched on demand) */
  uint32_t saber_ctas;     /* CTAs that take only Saber work (0 = none): Saber latency never waits on FrodoKEM */
  uint32_t warp_max;       /* a thread-level stage with at most this many ready instances runs a warp per instance */
  uint64_t scratch_bytes;  /* device scratch for the records of requests in flight (0 = max_inflight FrodoKEM records) */
  const uint8_t *coin_key; /* NULL, or 32 bytes: keypair / encaps requests with in0 NULL draw their coins on the device,
                              SHAKE256(key || LE64(ticket) || "kp" / "enc") truncated to the scheme's coin length */
} dpkem_service_config;
/* Defaults: 16384 slots, idle 1000 ms, no Saber-only CTAs, warp_max 32, default scratch, no key. */
int dpkem_service_default_config(dpkem_service_config *cfg);
/* cfg NULL = the defaults.  Device memory (ring, queues, scratch) counts against the context's budget. */
int dpkem_service_open(dpkem_ctx *ctx, int form, const dpkem_service_config *cfg, dpkem_service **out);
/* Accepts a prefix of reqs: *accepted requests with tickets *first_ticket, *first_ticket + 1, ...
 * DPKEM_EAGAIN when none fits yet (poll, then resubmit). */
int dpkem_service_submit(dpkem_service *svc, size_t n, const dpkem_request *reqs, size_t *accepted,
                         uint64_t *first_ticket);
/* Up to max tickets completed since the previous poll, in the order they were seen. */
int dpkem_service_poll(dpkem_service *svc, uint64_t *tickets, size_t max, size_t *n_done);
/* Waits until every accepted request has completed (DPKEM_ETIMEOUT after timeout_ms). */
int dpkem_service_drain(dpkem_service *svc, uint32_t timeout_ms);
/* Counters: tickets issued, tickets completed in order, launches so far, launch running now. */
int dpkem_service_stats(dpkem_service *svc, uint64_t *submitted, uint64_t *completed, uint64_t *launches,
                        int *running);
/* Diagnostic counters since open (or the last reset), up to n of them: for each queue
 * q = (scheme * 3 + op) * 4 + stage, out[4q .. 4q+3] = claims, instances, claims run as a warp
 * per instance, busy ns (claim to hand-off, summed over CTAs); then out[240] = CTA idle ns,
 * out[241] = admissions, out[242] = requests admitted, out[243] = claims lost to another CTA.  Counters are updated while the launch
 * runs; a read during traffic is a snapshot. */
int dpkem_service_counters(dpkem_service *svc, uint64_t *out, size_t n, int reset);
/* Drains (30 s at most), ends the launch and frees the service. */
int dpkem_service_close(dpkem_service *svc);

/* Seeded synthetic coins: out[i] = SHAKE256(00 01 .. 1F || LE64(first + i) || tag, len), len <= 136,
 * strlen(tag) <= 16.  Same flag semantics as the batched operations. */
int dpkem_coins(dpkem_ctx *ctx, size_t n, size_t len, uint64_t first, const char *tag, uint8_t *out,
                unsigned flags, void *stream);

/* Wait for `stream` (NULL = context stream) and report a device-side timeout, if any. */
int dpkem_sync(dpkem_ctx *ctx, void *stream);

/* Stage timing: when enabled, each batched call records CUDA events on its stream
 * between the kernels of its launch chain; dpkem_profile_read() waits for them and
 * returns the number of stages of the last call (its last chunk), filling stage_ms.
 * Frodo enc: prologue, S'A product, final hash; dec: W/decode, prologue, product, hash.
 * Saber enc: prologue, product, finish; dec: inner product, prologue, product, finish. */
int dpkem_profile(dpkem_ctx *ctx, int enable);
int dpkem_profile_read(dpkem_ctx *ctx, float *stage_ms, int max_stages);

/* Integer-pipe roofline probes on the context's device: 32-bit LOP3/SHF ops per second
 * in Keccak's instruction mix, and register-resident Keccak-f[1600] permutations per second. */
int dpkem_probe_int_peaks(dpkem_ctx *ctx, double *int_ops_per_s, double *keccak_per_s);
/* int8 tensor-core peak of this GPU: one CTA per SM issuing back-to-back 128 x 256 x 32
 * tcgen05.mma kind::i8 (u8 x s8, s32 accumulators in TMEM); int8 multiply-adds per second. */
int dpkem_probe_i8_mma_peak(dpkem_ctx *ctx, double *macs_per_s);

/* ---- FrodoKEM batches under one key (device pointers, enqueued on `stream`) ----
 * Many encapsulations to one public key, or many decapsulations with one secret key (a
 * server decapsulating under its own key): the n instances share the key's matrix A, so it
 * can be expanded once (dpkem_frodo_expand_a: A as 976 x 976 little-endian u16, row-major,
 * 1,905,152 bytes, 16-byte aligned) and read from memory instead of being regenerated by each
 * instance (amat NULL keeps the generation).  With amat and DPKEM_FORM_TC the products of all
 * instances run as one int8 tcgen05 GEMM (S' of every instance times [A | B]); the other forms
 * read A's rows per instance.  Encaps also hashes pk once.  Byte
 * layouts are the batched calls'; results equal dpkem_enc_batch / dpkem_dec_batch with the
 * key repeated n times.  dpkem_sync() reports device-side errors.  No counterpart in the
 * reference, whose instances all regenerate A (FrodoKEM976-GPU/src/cuda_kernel.cu:172-173,
 * :302-303). */
int dpkem_frodo_expand_a(dpkem_ctx *ctx, int scheme, const uint8_t *pk, uint16_t *amat, void *stream);
int dpkem_frodo_enc_shared(dpkem_ctx *ctx, int scheme, int form, size_t n, const uint8_t *coins, const uint8_t *pk,
                           const uint16_t *amat, uint8_t *ct, uint8_t *ss, void *stream);
int dpkem_frodo_dec_shared(dpkem_ctx *ctx, int scheme, int form, size_t n, const uint8_t *ct, const uint8_t *sk,
                           const uint16_t *amat, uint8_t *ss, void *stream);

/* Keccak-f[1600] in each lanes-per-state layout the sponge stages use (1: a thread per state,
 * 2: a bit-interleaved lane pair, 5: five lanes of a warp, 25: a warp per state): `perms` permutations
 * applied to each of n states (25 little-endian 64-bit lanes each, device pointers, 8-byte
 * aligned); returns when done.  No counterpart in the reference (its permutation is
 * KeccakF1600_StatePermute, FrodoKEM976-GPU/src/shake.cu:66-331, one thread per state). */
int dpkem_keccak_f1600_lanes(dpkem_ctx *ctx, int lanes, size_t n, const uint64_t *in, uint64_t *out, int perms);
/* Device time (ms, CUDA events) of `perms` dependent permutations on each of `states` states
 * in the given layout: the latency of a sponge chain per layout and batch size. */
int dpkem_probe_keccak_chain(dpkem_ctx *ctx, int lanes, int states, int perms, double *ms);

/* Saber encapsulation that allocates no device memory (no counterpart in the reference).
 * For callers that may not call cudaMalloc on their request path (allocator calls are
 * forbidden there, all device memory belongs to a host framework, or a fixed memory
 * quota applies).  Scratch is a fixed __device__ array inside the library, sized for
 * DPKEM_SABER_ENC_STATIC_MAX instances (about 3.9 MB, held on every GPU that loads the
 * library until exit); n above that returns DPKEM_EINVAL.  coins, pk, ct, ss are device
 * pointers (8-byte aligned) on the device that owns `stream`, laid out as in
 * dpkem_enc_batch; stream NULL is the current device's legacy default stream.  The call
 * returns when the work has finished and records its status for dpkem_last_status().
 * The first call on each device (and again after a device reset) resolves the array's
 * address on that device (make it before any stream capture).  All calls on a device
 * share the array: the library serialises its own calls per device, and work that
 * overlaps them on the GPU would race. */
#define DPKEM_SABER_ENC_STATIC_MAX 512
int dpkem_saber_enc_batch_static(int scheme, int form, size_t n, const uint8_t *coins, const uint8_t *pk,
                                 uint8_t *ct, uint8_t *ss, void *stream);

/* Runtime tuning knobs (process-wide): "thread_block" (block size of the thread-per-instance
 * kernels, multiple of 32, <= 256), "mixed_frodo_task" / "mixed_pair_task" /
 * "mixed_thread_task" (instances per thread-level task in mixed batches), "pipe_chunks"
 * (chunks, one stream each, of a pipelined host-buffer batch, <= 16), "pipe_priority" (0/1:
 * chunk streams with descending priorities, so earlier chunks finish first),
 * "saber_pair_max" (Keccak lanes per state in the Saber prologue: batches of up to this many
 * instances run GenMatrix on two lanes per state, larger ones on one; 0 = never).  Chosen by
 * dpcrypto_b200/autotune.py and stored in dpcrypto_b200/tuning.json. */
int dpkem_set_tuning(const char *key, int value);
/* Current value of a knob (DPKEM_EINVAL for an unknown key). */
int dpkem_get_tuning(const char *key, int *value);

const char *dpkem_strerror(int status);
/* Status of the last call made by this thread (the compatibility shims return void). */
int dpkem_last_status(void);

/* ---- Reference-compatible shims (process-wide default context on device 0) ---- */
void dpkem_set_compat_batch(size_t n);     /* default 768, the reference's BLOCK / BATCH */
void dpkem_set_compat_saber_level(int l);  /* default 3, the reference's SABER_L */
void dpkem_set_compat_form(int form);      /* default DPKEM_FORM_TC */
/* Keypair coins come from dpkem_coins(i, "kp"), encaps coins from dpkem_coins(i, "enc"). */
void frodoKEMKeypair(uint8_t *h_pk, uint8_t *h_sk);
void frodoKEMEncap(uint8_t *ct, uint8_t *ss, const uint8_t *pk);
void frodoKEMDecap(uint8_t *ss, const uint8_t *ct, const uint8_t *sk);
/* Reference: keys from tv.h, overwriting h_pk / h_sk.  Here caller data is used as given.
 * mode 0 = dp4a, 1 = INT32, 2 = tcgen05; any other mode computes nothing and records
 * DPKEM_EINVAL (the reference runs its INT32 path for every mode other than 0). */
void saber_enc(uint8_t mode, uint8_t *h_k, uint8_t *h_pk, uint8_t *h_c);
void saber_dec(uint8_t mode, uint8_t *h_c, uint8_t *h_pk, uint8_t *h_sk, uint8_t *h_k);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif
