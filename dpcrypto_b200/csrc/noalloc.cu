// Saber encapsulation that allocates no device memory.
//
// Who needs this: callers that are not allowed to call cudaMalloc at request time —
// for example a latency-critical key-exchange front end that forbids allocator calls
// (and their implicit device synchronisation) on the request path, code embedded in a
// host framework that owns all device memory and hands out only buffers it allocated,
// or a process running under a fixed device-memory quota.  The regular entry points
// grow a per-context arena with cudaMalloc on first use; this one never does.
//
// How: the per-instance scratch records that the Saber launch chain needs live in one
// file-scope __device__ array of fixed size (DPKEM_SABER_ENC_STATIC_MAX instances of the
// largest Saber record, about 3.9 MB), which every GPU that loads the library keeps until
// process exit.  Host code cannot use the array's name as a device address, so on the
// first call on each device (with that device current) the address is fetched once with
// cudaGetSymbolAddress, checked, cached per device and then passed to the kernels.
// All calls on a device share the array and it keeps the previous call's contents;
// everything the chain reads is written earlier in the same call, and the one word that
// must start at zero (the device error word) is cleared at the start of every call.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/dpkem.h"
#include "common.cuh"
#include "saber_dev.cuh"

namespace {

constexpr size_t kMaxInst = DPKEM_SABER_ENC_STATIC_MAX;
constexpr size_t kRecord = dpkem::sdev::Scr<4>::BYTES;  // largest Saber scratch record (FireSaber)
static_assert(dpkem::sdev::Scr<4>::BYTES >= dpkem::sdev::Scr<3>::BYTES &&
                  dpkem::sdev::Scr<4>::BYTES >= dpkem::sdev::Scr<2>::BYTES,
              "FireSaber has the largest record");
constexpr size_t kScratchBytes = kMaxInst * kRecord;
constexpr size_t kErrOffset = kScratchBytes + kMaxInst * 4;  // after the per-instance fail words

static __device__ __align__(256) uint8_t g_saber_enc_scratch[kErrOffset + 256];

constexpr int kMaxDevices = 64;
std::mutex g_mu;  // serialises calls, so two calls never use the array at the same time
uint8_t *g_addr[kMaxDevices] = {};

bool aligned8(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 7u) == 0; }

}  // namespace

extern "C" int dpkem_saber_enc_batch_static(int scheme, int form, size_t n, const uint8_t *coins, const uint8_t *pk,
                                            uint8_t *ct, uint8_t *ss, void *stream) {
  if (scheme < DPKEM_LIGHTSABER || scheme > DPKEM_FIRESABER) return DPKEM_EINVAL;
  if (form != DPKEM_FORM_DP4A && form != DPKEM_FORM_TC && form != DPKEM_FORM_INT32) return DPKEM_EINVAL;
  if (n > kMaxInst) return DPKEM_EINVAL;  // larger batches: split them, or use dpkem_enc_batch
  if (n == 0) return DPKEM_OK;
  if (!coins || !pk || !ct || !ss || !aligned8(coins) || !aligned8(pk) || !aligned8(ct) || !aligned8(ss))
    return DPKEM_EINVAL;
  if (dpkem::saber_scratch_bytes(scheme) > kRecord) return DPKEM_EINVAL;
  std::lock_guard<std::mutex> lock(g_mu);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return DPKEM_ECUDA;
  }
  if (!g_addr[dev]) {  // first call on this device: resolve the array's device address
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, g_saber_enc_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return DPKEM_ECUDA;
    }
    g_addr[dev] = static_cast<uint8_t *>(p);
  }
  uint8_t *base = g_addr[dev];
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  dpkem::SaberBatch b{};
  b.n = static_cast<int>(n);
  b.level = scheme;
  b.coins = coins;
  b.pk = const_cast<uint8_t *>(pk);
  b.ct = ct;
  b.ss = ss;
  b.scr = base;
  b.fail = reinterpret_cast<uint32_t *>(base + kScratchBytes);
  b.err = reinterpret_cast<uint32_t *>(base + kErrOffset);
  b.timer = nullptr;
  if (cudaMemsetAsync(b.err, 0, 4, st) != cudaSuccess) {
    cudaGetLastError();
    return DPKEM_ECUDA;
  }
  if (dpkem::saber_enc(b, form, st) != cudaSuccess) {
    cudaGetLastError();
    return DPKEM_ECUDA;
  }
  uint32_t err = 0;
  if (cudaMemcpyAsync(&err, b.err, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    cudaGetLastError();
    return DPKEM_ECUDA;
  }
  return err ? DPKEM_ETIMEOUT : DPKEM_OK;
}
