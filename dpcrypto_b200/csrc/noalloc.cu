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
// process exit.  Host code cannot use the array's name as a device address, so the first
// call on each device (made with that device current: the device that owns `stream`)
// fetches the address with cudaGetSymbolAddress, checks it and caches it for that device
// together with the CUDA context it belongs to; a later call under another context (after
// cudaDeviceReset the module is loaded again, at a new address) resolves it again.
// All calls on a device share the array and it keeps the previous call's contents;
// everything the chain reads is written earlier in the same call, and the one word that
// must start at zero (the device error word) is cleared at the start of every call.
// Calls on one device are serialised by a per-device lock; calls on different devices
// run independently.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/dpkem.h"
#include "common.cuh"
#include "ctx.h"
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
std::mutex g_mu[kMaxDevices];  // one lock per device: two calls never use one device's array at once
struct Resolved {
  void *ctx = nullptr;  // CUDA context the address belongs to
  uint8_t *addr = nullptr;
};
Resolved g_addr[kMaxDevices];

bool aligned8(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 7u) == 0; }

// cuCtxGetCurrent through the runtime's driver entry point (no link against libcuda).
using CtxGetCurrent = int (*)(void **);
CtxGetCurrent ctx_get_current() {
  static const CtxGetCurrent fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      p = nullptr;
    }
    return reinterpret_cast<CtxGetCurrent>(p);
  }();
  return fn;
}

// Makes `dev` current for the lifetime of the guard and restores the caller's device after.
struct DeviceGuard {
  int prev = -1;
  bool ok = false;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      cudaGetLastError();
      return;
    }
    ok = prev == dev || cudaSetDevice(dev) == cudaSuccess;
    if (!ok) cudaGetLastError();
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

// Device address of the scratch array on the current device `dev`, resolved once per
// device and context.
uint8_t *scratch_address(int dev) {
  const CtxGetCurrent get = ctx_get_current();
  void *ctx = nullptr;
  Resolved &r = g_addr[dev];
  if (r.addr && get && get(&ctx) == 0 && ctx && r.ctx == ctx) return r.addr;
  void *p = nullptr;
  if (cudaGetSymbolAddress(&p, g_saber_enc_scratch) != cudaSuccess || !p) {
    cudaGetLastError();
    return nullptr;
  }
  // The lookup has made the device's context current if it was not yet; without a
  // context handle (no driver entry point) r.ctx stays null and the address is fetched
  // on every call.
  ctx = nullptr;
  r.ctx = get && get(&ctx) == 0 ? ctx : nullptr;
  r.addr = static_cast<uint8_t *>(p);
  return r.addr;
}

int run(int scheme, int form, size_t n, const uint8_t *coins, const uint8_t *pk, uint8_t *ct, uint8_t *ss,
        void *stream) {
  if (scheme < DPKEM_LIGHTSABER || scheme > DPKEM_FIRESABER) return DPKEM_EINVAL;
  if (form != DPKEM_FORM_DP4A && form != DPKEM_FORM_TC && form != DPKEM_FORM_INT32) return DPKEM_EINVAL;
  if (n > kMaxInst) return DPKEM_EINVAL;  // larger batches: split them, or use dpkem_enc_batch
  if (n == 0) return DPKEM_OK;
  if (!coins || !pk || !ct || !ss || !aligned8(coins) || !aligned8(pk) || !aligned8(ct) || !aligned8(ss))
    return DPKEM_EINVAL;
  if (dpkem::saber_scratch_bytes(scheme) > kRecord) return DPKEM_EINVAL;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int dev = 0;
  if (cudaStreamGetDevice(st, &dev) != cudaSuccess) {  // NULL: the current device's legacy stream
    cudaGetLastError();
    return DPKEM_ECUDA;
  }
  if (dev < 0 || dev >= kMaxDevices) return DPKEM_EINVAL;
  std::lock_guard<std::mutex> lock(g_mu[dev]);
  DeviceGuard on(dev);
  if (!on.ok) return DPKEM_ECUDA;
  uint8_t *base = scratch_address(dev);
  if (!base) return DPKEM_ECUDA;
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

}  // namespace

extern "C" int dpkem_saber_enc_batch_static(int scheme, int form, size_t n, const uint8_t *coins, const uint8_t *pk,
                                            uint8_t *ct, uint8_t *ss, void *stream) {
  return dpkem::abi::set_status(run(scheme, form, n, coins, pk, ct, ss, stream));
}
