// Shared definitions for the batched KEM kernels: scheme parameters, batch
// descriptors and launcher prototypes.  Host code (abi.cu) fills the descriptors
// with device pointers to caller data and to the context's scratch arena.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace dpkem {

// ---- FrodoKEM-976-SHAKE (FrodoKEM976-GPU/include/params.h:9-25, api.h:7-10) ----
namespace frodo {
constexpr int N = 976, NBAR = 8, SEEDA = 16, LENS = 24, LENSE = 24, LENMU = 24, LENPKH = 24;
constexpr int PK = 15632, SK = 31296, CT = 15744, SS = 24, KP_COINS = 64, ENC_COINS = 24;
constexpr int PKB = N * NBAR * 2;               // packed B / B' bytes (15616)
constexpr int RW = (2 * N + NBAR) * NBAR;       // sampled words per instance (15680)
constexpr int SK_S = LENS + PK;                 // offset of S^T in sk (15656)
constexpr int SK_PKH = SK_S + PKB;              // offset of H(pk) in sk (31272)
constexpr int ROWS_PAD = 992;                   // 31 chunks of 32 rows
}  // namespace frodo

// ---- Saber (SABER-GPU/include/params.h:4-48) ----
namespace saber {
constexpr int N = 256, EQ = 13, EP = 10;
struct Params {
  int l, mu, et;
  int polyvec, polyveccomp, pk, sk, ct, coins_poly;
};
__host__ __device__ constexpr Params params(int level) {
  const int l = level, mu = level == 2 ? 10 : level == 3 ? 8 : 6, et = level == 2 ? 3 : level == 3 ? 4 : 6;
  const int polyvec = l * EQ * N / 8, polyveccomp = l * EP * N / 8;
  const int pk = polyveccomp + 32;
  return Params{l, mu, et, polyvec, polyveccomp, pk, polyvec + pk + 64, polyveccomp + et * N / 8, mu * N / 8};
}
}  // namespace saber

enum Op : int { OP_KEYPAIR = 0, OP_ENC = 1, OP_DEC = 2 };

// Runtime tuning knobs (set through dpkem_set_tuning; chosen by dpcrypto_b200/autotune.py).
struct Tuning {
  int thread_block = 64;        // block size of the thread-per-instance kernels
  int mixed_frodo_task = 256;   // instances per Frodo thread-level task in a mixed batch
  int mixed_pair_task = 128;    // instances per two-role prologue task (two threads each)
  int mixed_thread_task = 256;  // instances per other thread-level task
  // groups of up to this many requests run their sponge stages on a warp each (0: never).
  // Off: a planned batch of 32 mixed requests took 12.2 ms with warp tasks, 4.5 ms without
  int mixed_warp_max = 0;
  int pipe_chunks = 4;          // chunks (one stream each) of a pipelined host-mode batch, <= 16
  int pipe_priority = 1;        // 1: chunk streams get descending priorities (earlier chunks finish first)
  int saber_pair_max = 6144;    // largest Saber batch whose prologue runs GenMatrix on lane pairs (0: never)
  int saber_warp_max = 512;     // largest Saber batch whose prologue sponges run on a warp per state (0: never)
  int saber_finish_warp_max = 1024;  // the same for the encaps / keypair finish
  int saber_five_max = 0;       // largest Saber batch whose prologue sponges run on five lanes per state (0: never)
  int saber_finish_five_max = 0;  // the same for the encaps / keypair finish
  int frodo_warp_max = 1024;    // largest Frodo batch whose prologues run on a warp per state (0: never)
  int frodo_ss_warp_max = 1024; // the same for H(pk) and the final hash
  int frodo_five_max = 0;       // largest Frodo batch whose prologues run on five lanes per state (0: never)
  int frodo_ss_five_max = 0;    // the same for H(pk) and the final hash
  int saber_tc_ctas_per_sm = 0; // persistent Saber tensor-core product CTAs per SM (0: a CTA per instance)
};
Tuning &tuning();

// Optional per-stage timing: when non-null, a launcher records ev[k] on its stream
// before its k-th stage and ev[nstages] after the last one.
struct StageTimer {
  static constexpr int kMax = 8;
  cudaEvent_t ev[kMax + 1];
  int n = 0;
  void mark(cudaStream_t st) {
    if (n <= kMax) cudaEventRecord(ev[n++], st);
  }
};
enum Form : int { FORM_DP4A = 0, FORM_INT32 = 1, FORM_TC = 2 };

struct FrodoBatch {
  int n;
  int aes;               // 0: FrodoKEM-976-SHAKE, 1: FrodoKEM-976-AES (A rows from AES-128)
  const uint8_t *coins;  // keypair [n][64] = s||seedSE||z; enc [n][24] = mu
  uint8_t *pk;           // [n][15632]
  uint8_t *sk;           // [n][31296]
  uint8_t *ct;           // [n][15744]
  uint8_t *ss;           // [n][24]
  uint16_t *rw;          // scratch [n][15680]: sampled S'|E'|E'' (keypair: S^T|E)
  uint8_t *kk;           // scratch [n][24]: k (enc) or k' (dec)
  uint8_t *mu;           // scratch [n][24]: decoded mu' (dec)
  uint32_t *fail;        // scratch [n]: nonzero when the re-encryption differs (dec)
  uint2 *hs;             // scratch [n][25]: SHAKE256 state after absorbing ct's full blocks (dec)
  uint32_t *err;         // device error word (DEV_ERR_*)
  StageTimer *timer;     // optional
  // One key for the whole batch (enc: one pk, dec: one sk): pk / sk are not strided, A may
  // come expanded from memory (amat, 976 x 976 LE u16, rows of 1952 bytes) instead of being
  // regenerated by every instance, and encaps reads H(pk) from pkh (24 bytes) when given.
  int shared;
  const uint16_t *amat;
  const uint8_t *pkh;
  // Shared key with A in memory, tensor-core form: the S'A and S'B products of all instances
  // run as one GEMM (frodo_gemm.cuh) on operand tiles prepared in these scratch buffers
  // ([A | B] limb tiles, fgemm::AB_BYTES; S' tiles, fgemm::s_bytes(n)); null: per-instance path.
  uint8_t *abt;
  uint8_t *stile;
};

struct SaberBatch {
  int n, level;
  const uint8_t *coins;  // keypair [n][96] = seedA||seed_s||z; enc [n][32]
  uint8_t *pk, *sk, *ct, *ss;
  uint8_t *scr;          // scratch [n][saber_scratch_bytes(level)]: XOF bytes, kr, m
  uint32_t *fail;        // scratch [n]
  uint32_t *err;         // device error word (DEV_ERR_*)
  StageTimer *timer;     // optional
};

struct CoinsBatch {
  int n;
  int len;               // bytes per instance, <= 136
  uint64_t first;        // index of the first instance
  uint8_t tag[16];
  int taglen;
  uint8_t *out;          // [n][len]
};

cudaError_t frodo_keypair(const FrodoBatch &b, int form, cudaStream_t st);
cudaError_t frodo_enc(const FrodoBatch &b, int form, cudaStream_t st);
cudaError_t frodo_dec(const FrodoBatch &b, int form, cudaStream_t st);
// Shared-key helpers: A of one public key (aes: the AES-128 variant) into amat (976 x 976
// LE u16), and H(pk) = SHAKE256(pk, 24) of one public key into out.
cudaError_t frodo_expand_a(int aes, const uint8_t *pk, uint16_t *amat, cudaStream_t st);
// Scratch of the shared-key tensor-core GEMM: [A | B] operand tiles, S' tiles for n instances.
size_t frodo_gemm_ab_bytes();
size_t frodo_gemm_s_bytes(size_t n);
cudaError_t frodo_pk_digest(const uint8_t *pk, uint8_t *out, cudaStream_t st);

cudaError_t saber_keypair(const SaberBatch &b, int form, cudaStream_t st);
cudaError_t saber_enc(const SaberBatch &b, int form, cudaStream_t st);
cudaError_t saber_dec(const SaberBatch &b, int form, cudaStream_t st);
size_t saber_scratch_bytes(int level);
cudaError_t coins_generate(const CoinsBatch &b, cudaStream_t st);
cudaError_t probe_int_peaks(cudaStream_t st, double *int_ops_per_s, double *keccak_per_s);
// keccak_lanes.cu: `perms` Keccak-f[1600] permutations on each of n states (25 LE lanes each)
// with 1, 2 or 5 lanes per state; and the device time of such a dependent chain.
cudaError_t keccak_lanes(int lanes, const uint64_t *in, uint64_t *out, int n, int perms, cudaStream_t st);
cudaError_t probe_keccak_chain(int lanes, int n, int perms, cudaStream_t st, double *ms);
// int8 tcgen05 MMA throughput (MACs/s) of the device; err receives DEV_ERR_TIMEOUT if the
// probe's bounded wait expires.
cudaError_t probe_i8_mma_peak(cudaStream_t st, uint32_t *err, double *macs_per_s);

namespace mixed {
struct Req {
  int32_t scheme, op;
  const uint8_t *in0, *in1;
  uint8_t *out0, *out1;
};
size_t plan_bytes(const Req *reqs, size_t n, size_t *ntasks_out);
size_t plan_struct_bytes();
// coin_key (32 bytes, may be null): keypair / encaps requests with in0 == null draw their
// coins on the device, SHAKE256(coin_key || LE64(coin_first + i) || "kp" / "enc").
// The request / task / index tables are written to `stage` (pinned host memory, at least
// plan_table_bytes) and uploaded with one asynchronous copy, the caller keeping `stage`
// untouched until that copy has run; without a stage they go through a pageable buffer
// and the call waits for the copy.
cudaError_t plan_build(const Req *reqs, size_t n, int form, int slots, uint8_t *arena, size_t arena_bytes,
                       uint32_t *err, cudaStream_t st, void *plan_out, const uint8_t *coin_key = nullptr,
                       uint64_t coin_first = 0, uint8_t *stage = nullptr, size_t stage_bytes = 0);
size_t plan_table_bytes(const Req *reqs, size_t n);
cudaError_t kernel_setup(int *grid);
cudaError_t plan_launch(const void *plan, size_t n, int grid, cudaStream_t st);
// Writes the wire-format response header before each request's first output (the request
// header sits before its first input) and zeroes the frame's tail padding;
// resp_bytes / payload_end [scheme * 3 + op] = response frame size / end of its payload.
cudaError_t frame_headers_launch(const void *plan, size_t n, const uint32_t *resp_bytes, const uint32_t *payload_end,
                                 cudaStream_t st);
int slots_for_device();
// Diagnostics: a kernel whose bounded wait cannot be satisfied (0: an mbarrier nothing
// arrives on; 1: a persistent-kernel dependency nothing completes; needs 16 KB of arena).
cudaError_t selftest_timeout(int which, uint8_t *arena, size_t arena_bytes, uint32_t *err, cudaStream_t st);
}  // namespace mixed

}  // namespace dpkem
