// Host-side state of a dpkem context and the helpers shared by the C-ABI sources
// (abi.cu: batched calls, mixed batches, graphs; frames.cu: the wire-format entry points).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <mutex>

#include "../../include/dpkem.h"
#include "common.cuh"

struct dpkem_ctx {
  int device = 0;
  size_t budget = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t last = nullptr;  // recorded after every launch chain that used the arena
  cudaStream_t pipe[16] = {};   // host-mode copy/compute pipeline, one stream per chunk
  cudaStream_t ppipe[16] = {};  // the same with descending priorities (chunk 0 highest)
  cudaEvent_t pev[16] = {};
  uint8_t *arena = nullptr;
  size_t arena_bytes = 0;
  uint32_t *d_err = nullptr;
  int max_ctas = 0;  // persistent launches use at most this many CTAs (0: two per SM)
  uint8_t *h_stage[16] = {};      // pinned plan-table images, one per pipeline slot
  size_t h_stage_bytes[16] = {};
  cudaEvent_t stage_ev[16] = {};  // recorded after each stage's last upload
  bool profile = false;
  dpkem::StageTimer timer;
  int timer_stages = 0;
  std::mutex mu;
};

namespace dpkem {
namespace abi {

constexpr size_t kAlign = 256;
constexpr int kPipeChunks = 16;  // most chunks (and streams) of a pipelined host-mode batch

inline size_t up(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

struct Sizes {
  size_t pk, sk, ct, ss, kpc, encc;
};

int set_status(int s);                      // records the calling thread's last status
bool scheme_sizes(int scheme, Sizes *z);    // object sizes of a scheme; false if unknown
int ensure_arena(dpkem_ctx *c, size_t bytes);  // grows the context's device arena
int cuda_status(cudaError_t e);             // DPKEM_OK or DPKEM_ECUDA (clears the error)
// Grid of this context's persistent launches: the device's resident CTAs, capped by max_ctas.
cudaError_t persistent_grid(const dpkem_ctx *c, int *grid);
// Pinned stage j of at least `bytes`, once its previous upload has run (nullptr if it
// cannot be allocated: the caller then uploads synchronously); stage_used records the
// upload just enqueued on st.
uint8_t *stage_for(dpkem_ctx *c, int j, size_t bytes);
void stage_used(dpkem_ctx *c, int j, cudaStream_t st);
// DPKEM_OK when every request names a known scheme and operation with the buffers it needs,
// aligned as the mixed entry points require (device_coins: keypair / encaps may omit coins).
int check_requests(size_t n, const dpkem_request *reqs, bool device_coins = false);

}  // namespace abi
}  // namespace dpkem
