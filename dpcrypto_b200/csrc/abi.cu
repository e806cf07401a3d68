// C ABI of libdpkem.so (declared in include/dpkem.h): contexts, the scratch arena,
// host<->device staging, chunking, status codes and the reference-compatible shims.
//
// The reference allocates, copies and frees device buffers inside every call
// (FrodoKEM976-GPU/src/cuda_kernel.cu:29-46, SABER-GPU/src/cuda_kernel.cu:36-58) and
// checks no CUDA status.  Here a context owns one device arena that grows only when a
// larger chunk is requested (never inside a steady-state loop), calls on one context
// are serialised on the device with an event so scratch is never shared by two
// in-flight chains, and every entry point returns a status.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/dpkem.h"
#include "common.cuh"
#include "ctx.h"

using namespace dpkem;

namespace dpkem {
Tuning &tuning() {
  static Tuning t;
  return t;
}
}  // namespace dpkem

namespace dpkem {
namespace abi {

thread_local int g_last_status = DPKEM_OK;

int set_status(int s) {
  g_last_status = s;
  return s;
}

bool scheme_sizes(int scheme, Sizes *z) {
  if (scheme == DPKEM_FRODO976 || scheme == DPKEM_FRODO976AES) {  // the variants share every size
    *z = {frodo::PK, frodo::SK, frodo::CT, frodo::SS, frodo::KP_COINS, frodo::ENC_COINS};
    return true;
  }
  if (scheme < 2 || scheme > 4) return false;
  const saber::Params p = saber::params(scheme);
  *z = {(size_t)p.pk, (size_t)p.sk, (size_t)p.ct, 32, 96, 32};
  return true;
}

// Per-instance bytes of scratch and, in host mode, of device staging for each op.
size_t scratch_per_instance(int scheme) {
  if (scheme <= DPKEM_FRODO976AES) return (size_t)frodo::RW * 2 + 24 + 24 + 4 + 200 + 80;
  return saber_scratch_bytes(scheme) + 4 + 16;
}

size_t staging_per_instance(int scheme, int op) {
  Sizes z;
  scheme_sizes(scheme, &z);
  switch (op) {
    case OP_KEYPAIR: return z.kpc + z.pk + z.sk;
    case OP_ENC: return z.pk + z.encc + z.ct + z.ss;
    default: return z.ct + z.sk + z.ss;
  }
}

size_t chunk_for(dpkem_ctx *c, int scheme, int op, bool host) {
  const size_t per = scratch_per_instance(scheme) + (host ? staging_per_instance(scheme, op) : 0) + 8 * kAlign / 64;
  const size_t usable = c->budget > (64u << 20) ? c->budget - (64u << 20) : c->budget / 2;
  return std::max<size_t>(1, usable / per);
}

// Growing the arena frees the old one (cudaFree waits for the whole device, other
// contexts' work included), so growth is geometric (at least 1.5x, within the budget) and
// callers on a latency path reserve the arena up front (dpkem_ctx_reserve).
int ensure_arena(dpkem_ctx *c, size_t bytes) {
  if (bytes <= c->arena_bytes) return DPKEM_OK;
  if (bytes > c->budget) return DPKEM_ENOMEM;
  const size_t want = std::min(c->budget, std::max(bytes, c->arena_bytes + c->arena_bytes / 2));
  if (c->arena) {
    // c->last follows every launch that used the arena, on whichever stream it ran
    cudaEventSynchronize(c->last);
    cudaFree(c->arena);
    c->arena = nullptr;
    c->arena_bytes = 0;
  }
  if (cudaMalloc(&c->arena, want) != cudaSuccess) {
    cudaGetLastError();
    return DPKEM_ENOMEM;
  }
  c->arena_bytes = want;
  return DPKEM_OK;
}

int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return DPKEM_OK;
  cudaGetLastError();
  return DPKEM_ECUDA;
}

cudaError_t persistent_grid(const dpkem_ctx *c, int *grid) {
  const cudaError_t e = mixed::kernel_setup(grid);
  if (e == cudaSuccess && c->max_ctas > 0) *grid = std::min(*grid, c->max_ctas);
  return e;
}

uint8_t *stage_for(dpkem_ctx *c, int j, size_t bytes) {
  if (c->stage_ev[j]) cudaEventSynchronize(c->stage_ev[j]);  // its previous upload has been read
  if (c->h_stage_bytes[j] < bytes) {
    if (c->h_stage[j]) cudaFreeHost(c->h_stage[j]);
    const size_t want = std::max({bytes, c->h_stage_bytes[j] + c->h_stage_bytes[j] / 2, (size_t)1 << 20});
    if (cudaHostAlloc(&c->h_stage[j], want, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      c->h_stage[j] = nullptr;
      c->h_stage_bytes[j] = 0;
      return nullptr;
    }
    c->h_stage_bytes[j] = want;
  }
  return c->h_stage[j];
}

void stage_used(dpkem_ctx *c, int j, cudaStream_t st) { cudaEventRecord(c->stage_ev[j], st); }

}  // namespace abi
}  // namespace dpkem

using namespace dpkem::abi;

namespace {

constexpr size_t kPipeChunkMin = 256;  // smallest chunk of a host-mode pipeline
constexpr size_t kDefaultBudget = 8ull << 30;

struct Carver {
  uint8_t *base;
  size_t off = 0;
  template <typename T>
  T *take(size_t bytes) {
    T *p = reinterpret_cast<T *>(base + off);
    off += up(bytes);
    return p;
  }
};

// Layout of one chunk's arena: scratch first, then (host mode) staging.
size_t arena_need(int scheme, int op, size_t chunk, bool host) {
  size_t s = 0;
  if (scheme <= DPKEM_FRODO976AES) {
    s += up(chunk * frodo::RW * 2) + up(chunk * 24) * 2 + up(chunk * 4) + up(chunk * 200);
  } else {
    s += up(chunk * saber_scratch_bytes(scheme)) + up(chunk * 4);
  }
  if (host) {
    Sizes z;
    scheme_sizes(scheme, &z);
    switch (op) {
      case OP_KEYPAIR: s += up(chunk * z.kpc) + up(chunk * z.pk) + up(chunk * z.sk); break;
      case OP_ENC: s += up(chunk * z.pk) + up(chunk * z.encc) + up(chunk * z.ct) + up(chunk * z.ss); break;
      default: s += up(chunk * z.ct) + up(chunk * z.sk) + up(chunk * z.ss); break;
    }
  }
  return s;
}

// Device buffers: pk and ct arrays must be 16-byte aligned (the Frodo stages move 16-byte
// vectors of them), coins, sk and ss arrays 8-byte aligned (64-bit lane loads/stores).
bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }
bool aligned8(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 7u) == 0; }

// Alignment check of an operation's buffers in argument order (see run_op).
bool op_aligned(int op, const void *in0, const void *in1, const void *out0, const void *out1) {
  switch (op) {
    case OP_KEYPAIR: return aligned8(in0) && aligned16(out0) && aligned8(out1);             // coins, pk, sk
    case OP_ENC: return aligned8(in0) && aligned16(in1) && aligned16(out0) && aligned8(out1);  // coins, pk, ct, ss
    default: return aligned16(in0) && aligned8(in1) && aligned8(out0);                     // ct, sk, ss
  }
}

// Runs op on n instances.  in0/in1/out0/out1 follow the op's argument order:
//   keypair: in0 = coins, out0 = pk, out1 = sk
//   enc:     in0 = coins, in1 = pk, out0 = ct, out1 = ss
//   dec:     in0 = ct, in1 = sk, out0 = ss
int run_op(dpkem_ctx *c, int scheme, int form, int op, size_t n, const uint8_t *in0, const uint8_t *in1, uint8_t *out0,
           uint8_t *out1, unsigned flags, void *stream) {
  Sizes z;
  if (!c || !scheme_sizes(scheme, &z)) return DPKEM_EINVAL;
  if (form != DPKEM_FORM_DP4A && form != DPKEM_FORM_TC && form != DPKEM_FORM_INT32) return DPKEM_EINVAL;
  if (n == 0) return DPKEM_OK;
  if (n > (size_t)INT32_MAX) return DPKEM_EINVAL;
  if (!in0 || !out0 || (op != OP_KEYPAIR && !in1) || (op != OP_DEC && !out1)) return DPKEM_EINVAL;
  const bool dev = (flags & DPKEM_FLAG_DEVICE_PTRS) != 0;
  if (dev && !op_aligned(op, in0, in1, out0, out1)) return DPKEM_EINVAL;
  std::lock_guard<std::mutex> lock(c->mu);
  if (cudaSetDevice(c->device) != cudaSuccess) return cuda_status(cudaErrorInvalidDevice);
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c->stream;
  // Host-mode batches of at least two minimum chunks, when the budget holds the whole batch,
  // run as a pipeline: up to pipe_chunks chunks, each on its own stream with its own arena region,
  // all in flight at once.  The copies of later chunks and their latency-bound first stages
  // then overlap the long kernels of earlier chunks.  With three or more chunks the first and
  // the last are a quarter of the others: the first upload and the last download are the
  // copies that no kernel overlaps.
  size_t chunk = std::min(n, chunk_for(c, scheme, op, !dev));
  int npipe = 1;
  size_t edge = 0;  // pipelined: size of the first and the last chunk (0: all equal)
  if (!dev && !c->profile && n >= 2 * kPipeChunkMin) {
    const int want = (int)std::min<size_t>(std::min(tuning().pipe_chunks, kPipeChunks), n / kPipeChunkMin);
    size_t each = (n + want - 1) / want, e = 0;
    if (want >= 3) {
      const size_t w = 2 + 4 * (size_t)(want - 2);  // weights 1, 4, ..., 4, 1
      e = std::max<size_t>(1, n / w);
      each = (n - 2 * e + want - 3) / (want - 2);
    }
    if (each * want <= chunk_for(c, scheme, op, true) && want > 1) {
      npipe = want;
      chunk = each;
      edge = e;
    }
  }
  const size_t per_pipe = (arena_need(scheme, op, chunk, !dev) + kAlign - 1) & ~(kAlign - 1);
  int rc = ensure_arena(c, per_pipe * npipe);
  if (rc) return rc;
  cudaError_t e = cudaStreamWaitEvent(st, c->last, 0);
  if (e != cudaSuccess) return cuda_status(e);
  cudaStream_t streams[kPipeChunks];
  for (int j = 0; j < kPipeChunks; j++) streams[j] = st;
  if (npipe > 1) {
    if ((e = cudaEventRecord(c->pev[0], st)) != cudaSuccess) return cuda_status(e);
    for (int j = 0; j < npipe; j++) {
      streams[j] = tuning().pipe_priority ? c->ppipe[j] : c->pipe[j];
      if ((e = cudaStreamWaitEvent(streams[j], c->pev[0], 0)) != cudaSuccess) return cuda_status(e);
    }
  }

  size_t in0_sz, in1_sz = 0, out0_sz, out1_sz = 0;
  switch (op) {
    case OP_KEYPAIR: in0_sz = z.kpc; out0_sz = z.pk; out1_sz = z.sk; break;
    case OP_ENC: in0_sz = z.encc; in1_sz = z.pk; out0_sz = z.ct; out1_sz = z.ss; break;
    default: in0_sz = z.ct; in1_sz = z.sk; out0_sz = z.ss; break;
  }
  size_t k = 0, m = 0;
  for (size_t first = 0; first < n; first += m, k++) {
    m = std::min(chunk, n - first);
    if (edge && (k == 0 || k + 1 == (size_t)npipe)) m = std::min(edge, n - first);
    const int j = (int)(k % (size_t)npipe);
    cudaStream_t sj = streams[j];
    Carver cv{c->arena + (size_t)j * per_pipe};
    const uint8_t *d_in0, *d_in1 = nullptr;
    uint8_t *d_out0, *d_out1 = nullptr;
    FrodoBatch fb{};
    SaberBatch sb{};
    if (scheme <= DPKEM_FRODO976AES) {
      fb.rw = cv.take<uint16_t>(chunk * frodo::RW * 2);
      fb.kk = cv.take<uint8_t>(chunk * 24);
      fb.mu = cv.take<uint8_t>(chunk * 24);
      fb.fail = cv.take<uint32_t>(chunk * 4);
      fb.hs = cv.take<uint2>(chunk * 200);
    } else {
      sb.scr = cv.take<uint8_t>(chunk * saber_scratch_bytes(scheme));
      sb.fail = cv.take<uint32_t>(chunk * 4);
    }
    if (dev) {
      d_in0 = in0 + first * in0_sz;
      d_in1 = in1 ? in1 + first * in1_sz : nullptr;
      d_out0 = out0 + first * out0_sz;
      d_out1 = out1 ? out1 + first * out1_sz : nullptr;
    } else {
      uint8_t *a = cv.take<uint8_t>(chunk * in0_sz);
      uint8_t *b = in1_sz ? cv.take<uint8_t>(chunk * in1_sz) : nullptr;
      d_out0 = cv.take<uint8_t>(chunk * out0_sz);
      d_out1 = out1_sz ? cv.take<uint8_t>(chunk * out1_sz) : nullptr;
      if ((e = cudaMemcpyAsync(a, in0 + first * in0_sz, m * in0_sz, cudaMemcpyHostToDevice, sj)) != cudaSuccess)
        return cuda_status(e);
      if (b && (e = cudaMemcpyAsync(b, in1 + first * in1_sz, m * in1_sz, cudaMemcpyHostToDevice, sj)) != cudaSuccess)
        return cuda_status(e);
      d_in0 = a;
      d_in1 = b;
    }
    StageTimer *tm = nullptr;
    if (c->profile) {
      c->timer.n = 0;
      tm = &c->timer;
    }
    fb.timer = tm;
    sb.timer = tm;
    if (scheme <= DPKEM_FRODO976AES) {
      fb.n = (int)m;
      fb.aes = scheme == DPKEM_FRODO976AES;
      fb.err = c->d_err;
      switch (op) {
        case OP_KEYPAIR:
          fb.coins = d_in0; fb.pk = d_out0; fb.sk = d_out1;
          e = frodo_keypair(fb, form, sj);
          break;
        case OP_ENC:
          fb.coins = d_in0; fb.pk = const_cast<uint8_t *>(d_in1); fb.ct = d_out0; fb.ss = d_out1;
          e = frodo_enc(fb, form, sj);
          break;
        default:
          fb.ct = const_cast<uint8_t *>(d_in0); fb.sk = const_cast<uint8_t *>(d_in1); fb.ss = d_out0;
          e = frodo_dec(fb, form, sj);
          break;
      }
    } else {
      sb.n = (int)m;
      sb.level = scheme;
      sb.err = c->d_err;
      switch (op) {
        case OP_KEYPAIR:
          sb.coins = d_in0; sb.pk = d_out0; sb.sk = d_out1;
          e = saber_keypair(sb, form, sj);
          break;
        case OP_ENC:
          sb.coins = d_in0; sb.pk = const_cast<uint8_t *>(d_in1); sb.ct = d_out0; sb.ss = d_out1;
          e = saber_enc(sb, form, sj);
          break;
        default:
          sb.ct = const_cast<uint8_t *>(d_in0); sb.sk = const_cast<uint8_t *>(d_in1); sb.ss = d_out0;
          e = saber_dec(sb, form, sj);
          break;
      }
    }
    if (e != cudaSuccess) return cuda_status(e);
    if (tm) c->timer_stages = tm->n - 1;
    if (!dev) {
      if ((e = cudaMemcpyAsync(out0 + first * out0_sz, d_out0, m * out0_sz, cudaMemcpyDeviceToHost, sj)) != cudaSuccess)
        return cuda_status(e);
      if (d_out1 &&
          (e = cudaMemcpyAsync(out1 + first * out1_sz, d_out1, m * out1_sz, cudaMemcpyDeviceToHost, sj)) != cudaSuccess)
        return cuda_status(e);
    }
  }
  if (npipe > 1) {  // join the pipeline back into the caller's stream
    for (int j = 0; j < npipe; j++) {
      if ((e = cudaEventRecord(c->pev[j], streams[j])) != cudaSuccess) return cuda_status(e);
      if ((e = cudaStreamWaitEvent(st, c->pev[j], 0)) != cudaSuccess) return cuda_status(e);
    }
  }
  if ((e = cudaEventRecord(c->last, st)) != cudaSuccess) return cuda_status(e);
  if (!dev) {
    uint32_t err = 0;
    if ((e = cudaMemcpyAsync(&err, c->d_err, 4, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return cuda_status(e);
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return cuda_status(e);
    if (err) {
      cudaMemsetAsync(c->d_err, 0, 4, st);
      cudaStreamSynchronize(st);
      return DPKEM_ETIMEOUT;
    }
  }
  return DPKEM_OK;
}

// Shared-key FrodoKEM batches (device pointers): op = OP_ENC runs n encapsulations to the
// one public key `key` (coins = in0, ct = out0, ss = out1), op = OP_DEC n decapsulations with
// the one secret key `key` (ct = in0, ss = out0).  amat: the key's A from
// dpkem_frodo_expand_a, or null (then every instance still generates its rows).  Encaps
// hashes pk once (H(pk) in the arena) instead of once per instance.
int run_shared(dpkem_ctx *c, int scheme, int form, int op, size_t n, const uint8_t *in0, const uint8_t *key,
               const uint16_t *amat, uint8_t *out0, uint8_t *out1, void *stream) {
  if (!c || (scheme != DPKEM_FRODO976 && scheme != DPKEM_FRODO976AES)) return DPKEM_EINVAL;
  if (form != DPKEM_FORM_DP4A && form != DPKEM_FORM_TC && form != DPKEM_FORM_INT32) return DPKEM_EINVAL;
  if (n == 0) return DPKEM_OK;
  if (n > (size_t)INT32_MAX || !in0 || !key || !out0 || (op == OP_ENC && !out1)) return DPKEM_EINVAL;
  if (!op_aligned(op, in0, key, out0, out1) || (amat && !aligned16(amat))) return DPKEM_EINVAL;
  std::lock_guard<std::mutex> lock(c->mu);
  if (cudaSetDevice(c->device) != cudaSuccess) return cuda_status(cudaErrorInvalidDevice);
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c->stream;
  const size_t chunk = std::min(n, chunk_for(c, scheme, op, false));
  // With A in memory, the tensor-core form runs the products as one GEMM on tiled operands.
  const bool gemm = amat && form == DPKEM_FORM_TC;
  const size_t tiles = gemm ? up(frodo_gemm_ab_bytes()) + up(frodo_gemm_s_bytes(chunk)) : 0;
  int rc = ensure_arena(c, arena_need(scheme, op, chunk, false) + kAlign + tiles);
  if (rc) return rc;
  cudaError_t e = cudaStreamWaitEvent(st, c->last, 0);
  if (e != cudaSuccess) return cuda_status(e);
  Carver cv{c->arena};
  FrodoBatch fb{};
  fb.rw = cv.take<uint16_t>(chunk * frodo::RW * 2);
  fb.kk = cv.take<uint8_t>(chunk * 24);
  fb.mu = cv.take<uint8_t>(chunk * 24);
  fb.fail = cv.take<uint32_t>(chunk * 4);
  fb.hs = cv.take<uint2>(chunk * 200);
  uint8_t *pkh = cv.take<uint8_t>(kAlign);
  if (gemm) {
    fb.abt = cv.take<uint8_t>(frodo_gemm_ab_bytes());
    fb.stile = cv.take<uint8_t>(frodo_gemm_s_bytes(chunk));
  }
  fb.aes = scheme == DPKEM_FRODO976AES;
  fb.err = c->d_err;
  fb.shared = 1;
  fb.amat = amat;
  if (c->profile) {
    c->timer.n = 0;
    fb.timer = &c->timer;
  }
  if (op == OP_ENC) {
    if ((e = frodo_pk_digest(key, pkh, st)) != cudaSuccess) return cuda_status(e);
    fb.pkh = pkh;
    fb.pk = const_cast<uint8_t *>(key);
  } else {
    fb.sk = const_cast<uint8_t *>(key);
  }
  for (size_t first = 0; first < n; first += chunk) {
    fb.n = (int)std::min(chunk, n - first);
    if (op == OP_ENC) {
      fb.coins = in0 + first * frodo::ENC_COINS;
      fb.ct = out0 + first * frodo::CT;
      fb.ss = out1 + first * frodo::SS;
      e = frodo_enc(fb, form, st);
    } else {
      fb.ct = const_cast<uint8_t *>(in0) + first * frodo::CT;
      fb.ss = out0 + first * frodo::SS;
      e = frodo_dec(fb, form, st);
    }
    if (e != cudaSuccess) return cuda_status(e);
    if (fb.timer) c->timer_stages = fb.timer->n - 1;
  }
  if ((e = cudaEventRecord(c->last, st)) != cudaSuccess) return cuda_status(e);
  return DPKEM_OK;
}

}  // namespace

namespace dpkem {
namespace abi {

// device_coins: keypair / encaps requests may leave in0 (coins) null.
int check_requests(size_t n, const dpkem_request *reqs, bool device_coins) {
  if (!reqs || n == 0 || n > (size_t)INT32_MAX) return DPKEM_EINVAL;
  alignas(16) static const uint8_t kAligned[16] = {};
  for (size_t i = 0; i < n; i++) {
    const dpkem_request &r = reqs[i];
    Sizes z;
    if (!scheme_sizes(r.scheme, &z) || r.op < 0 || r.op > 2) return DPKEM_EINVAL;
    const bool two_out = r.op != OP_DEC;
    const bool coins_ok = r.in0 || (device_coins && r.op != OP_DEC);
    if (!coins_ok || !r.out0 || (r.op != OP_KEYPAIR && !r.in1) || (two_out && !r.out1)) return DPKEM_EINVAL;
    if (!op_aligned(r.op, r.in0 ? r.in0 : kAligned, r.in1, r.out0, r.out1)) return DPKEM_EINVAL;
  }
  return DPKEM_OK;
}

}  // namespace abi
}  // namespace dpkem

extern "C" {

int dpkem_ctx_create(dpkem_ctx **out, int device, size_t hbm_budget_bytes) {
  if (!out) return set_status(DPKEM_EINVAL);
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    cudaGetLastError();
    return set_status(DPKEM_ECUDA);
  }
  if (cudaSetDevice(device) != cudaSuccess) return set_status(DPKEM_ECUDA);
  dpkem_ctx *c = new dpkem_ctx();
  c->device = device;
  c->budget = hbm_budget_bytes ? hbm_budget_bytes : kDefaultBudget;
  for (int k = 0; k <= StageTimer::kMax; k++) cudaEventCreate(&c->timer.ev[k]);
  for (int j = 0; j < kPipeChunks; j++) {
    cudaStreamCreateWithFlags(&c->pipe[j], cudaStreamNonBlocking);
    cudaEventCreateWithFlags(&c->pev[j], cudaEventDisableTiming);
    int least = 0, greatest = 0;  // numerically, greatest <= least
    cudaDeviceGetStreamPriorityRange(&least, &greatest);
    const int prio = greatest + (least - greatest) * j / (kPipeChunks - 1);
    cudaStreamCreateWithPriority(&c->ppipe[j], cudaStreamNonBlocking, prio);
    cudaEventCreateWithFlags(&c->stage_ev[j], cudaEventDisableTiming);
  }
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->last, cudaEventDisableTiming) != cudaSuccess ||
      cudaMalloc(&c->d_err, 4) != cudaSuccess || cudaMemset(c->d_err, 0, 4) != cudaSuccess) {
    cudaGetLastError();
    dpkem_ctx_destroy(c);
    return set_status(DPKEM_ECUDA);
  }
  *out = c;
  return set_status(DPKEM_OK);
}

int dpkem_ctx_reserve(dpkem_ctx *c, size_t bytes) {
  if (!c) return set_status(DPKEM_EINVAL);
  std::lock_guard<std::mutex> lock(c->mu);
  if (cudaSetDevice(c->device) != cudaSuccess) return set_status(cuda_status(cudaErrorInvalidDevice));
  return set_status(ensure_arena(c, bytes));
}

size_t dpkem_mixed_bytes(int scheme, size_t n) {
  Sizes z;
  if (!scheme_sizes(scheme, &z) || n == 0) return 0;
  std::vector<mixed::Req> rq(n, mixed::Req{scheme, OP_ENC, nullptr, nullptr, nullptr, nullptr});
  return mixed::plan_bytes(rq.data(), n, nullptr);
}

int dpkem_selftest_timeout(dpkem_ctx *c, int which) {
  if (!c || (which != 0 && which != 1)) return set_status(DPKEM_EINVAL);
  std::lock_guard<std::mutex> lock(c->mu);
  if (cudaSetDevice(c->device) != cudaSuccess) return set_status(cuda_status(cudaErrorInvalidDevice));
  int rc = ensure_arena(c, 16 << 10);
  if (rc) return set_status(rc);
  cudaStream_t st = c->stream;
  cudaError_t e = cudaStreamWaitEvent(st, c->last, 0);
  if (e == cudaSuccess) e = mixed::selftest_timeout(which, c->arena, c->arena_bytes, c->d_err, st);
  if (e == cudaSuccess) e = cudaEventRecord(c->last, st);
  uint32_t err = 0;
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaMemcpy(&err, c->d_err, 4, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return set_status(cuda_status(e));
  if (err) {
    cudaMemset(c->d_err, 0, 4);
    return set_status(DPKEM_ETIMEOUT);
  }
  return set_status(DPKEM_OK);
}

int dpkem_ctx_set_max_ctas(dpkem_ctx *c, int max_ctas) {
  if (!c || max_ctas < 0) return set_status(DPKEM_EINVAL);
  std::lock_guard<std::mutex> lock(c->mu);
  c->max_ctas = max_ctas;
  return set_status(DPKEM_OK);
}

int dpkem_ctx_destroy(dpkem_ctx *c) {
  if (!c) return set_status(DPKEM_EINVAL);
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->last) cudaEventSynchronize(c->last);
  if (c->arena) cudaFree(c->arena);
  if (c->d_err) cudaFree(c->d_err);
  if (c->last) cudaEventDestroy(c->last);
  for (int j = 0; j < kPipeChunks; j++) {
    if (c->pipe[j]) {
      cudaStreamSynchronize(c->pipe[j]);
      cudaStreamDestroy(c->pipe[j]);
    }
    if (c->ppipe[j]) {
      cudaStreamSynchronize(c->ppipe[j]);
      cudaStreamDestroy(c->ppipe[j]);
    }
    if (c->stage_ev[j]) {
      cudaEventSynchronize(c->stage_ev[j]);
      cudaEventDestroy(c->stage_ev[j]);
    }
    if (c->h_stage[j]) cudaFreeHost(c->h_stage[j]);
    if (c->pev[j]) cudaEventDestroy(c->pev[j]);
  }
  for (int k = 0; k <= StageTimer::kMax; k++)
    if (c->timer.ev[k]) cudaEventDestroy(c->timer.ev[k]);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return set_status(DPKEM_OK);
}

int dpkem_sizes(int scheme, size_t *pk, size_t *sk, size_t *ct, size_t *ss, size_t *kp_coins, size_t *enc_coins) {
  Sizes z;
  if (!scheme_sizes(scheme, &z)) return set_status(DPKEM_EINVAL);
  if (pk) *pk = z.pk;
  if (sk) *sk = z.sk;
  if (ct) *ct = z.ct;
  if (ss) *ss = z.ss;
  if (kp_coins) *kp_coins = z.kpc;
  if (enc_coins) *enc_coins = z.encc;
  return set_status(DPKEM_OK);
}

size_t dpkem_max_chunk(dpkem_ctx *c, int scheme) {
  Sizes z;
  if (!c || !scheme_sizes(scheme, &z)) return 0;
  return std::min({chunk_for(c, scheme, OP_KEYPAIR, true), chunk_for(c, scheme, OP_ENC, true),
                   chunk_for(c, scheme, OP_DEC, true)});
}

int dpkem_keypair_batch(dpkem_ctx *c, int scheme, int form, size_t n, const uint8_t *coins, uint8_t *pk, uint8_t *sk,
                        unsigned flags, void *stream) {
  return set_status(run_op(c, scheme, form, OP_KEYPAIR, n, coins, nullptr, pk, sk, flags, stream));
}

int dpkem_enc_batch(dpkem_ctx *c, int scheme, int form, size_t n, const uint8_t *coins, const uint8_t *pk, uint8_t *ct,
                    uint8_t *ss, unsigned flags, void *stream) {
  return set_status(run_op(c, scheme, form, OP_ENC, n, coins, pk, ct, ss, flags, stream));
}

int dpkem_dec_batch(dpkem_ctx *c, int scheme, int form, size_t n, const uint8_t *ct, const uint8_t *sk, uint8_t *ss,
                    unsigned flags, void *stream) {
  return set_status(run_op(c, scheme, form, OP_DEC, n, ct, sk, ss, nullptr, flags, stream));
}

static_assert(sizeof(dpkem_request) == sizeof(mixed::Req), "request layout");


static int mixed_batch(dpkem_ctx *c, int form, size_t n, const dpkem_request *reqs, const uint8_t *key,
                       uint64_t first, void *stream);

int dpkem_mixed_batch(dpkem_ctx *c, int form, size_t n, const dpkem_request *reqs, void *stream) {
  return mixed_batch(c, form, n, reqs, nullptr, 0, stream);
}

int dpkem_mixed_batch_keyed(dpkem_ctx *c, int form, size_t n, const dpkem_request *reqs, const uint8_t *key,
                            uint64_t first, void *stream) {
  if (!key) return set_status(DPKEM_EINVAL);
  return mixed_batch(c, form, n, reqs, key, first, stream);
}

static int mixed_batch(dpkem_ctx *c, int form, size_t n, const dpkem_request *reqs, const uint8_t *key,
                       uint64_t first, void *stream) {
  if (!c) return set_status(DPKEM_EINVAL);
  if (form != DPKEM_FORM_DP4A && form != DPKEM_FORM_TC && form != DPKEM_FORM_INT32) return set_status(DPKEM_EINVAL);
  if (n == 0) return set_status(DPKEM_OK);
  int rc = check_requests(n, reqs, key != nullptr);
  if (rc) return set_status(rc);
  std::lock_guard<std::mutex> lock(c->mu);
  cudaSetDevice(c->device);
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c->stream;
  const mixed::Req *mr = reinterpret_cast<const mixed::Req *>(reqs);
  const size_t need = mixed::plan_bytes(mr, n, nullptr);
  if ((rc = ensure_arena(c, need)) != DPKEM_OK) return set_status(rc);
  cudaError_t e = cudaStreamWaitEvent(st, c->last, 0);
  int grid = 0;
  if (e == cudaSuccess) e = persistent_grid(c, &grid);
  std::vector<uint8_t> plan(mixed::plan_struct_bytes());
  const size_t tb = mixed::plan_table_bytes(mr, n);
  uint8_t *stage = e == cudaSuccess ? stage_for(c, 0, tb) : nullptr;
  if (e == cudaSuccess)
    e = mixed::plan_build(mr, n, form, grid, c->arena, c->arena_bytes, c->d_err, st, plan.data(), key, first, stage,
                          stage ? c->h_stage_bytes[0] : 0);
  if (e == cudaSuccess && stage) stage_used(c, 0, st);
  if (e == cudaSuccess) e = mixed::plan_launch(plan.data(), n, grid, st);
  if (e == cudaSuccess) e = cudaEventRecord(c->last, st);
  return set_status(cuda_status(e));
}

struct dpkem_graph {
  dpkem_ctx *ctx = nullptr;
  uint8_t *mem = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

int dpkem_mixed_graph_destroy(dpkem_graph *g) {
  if (!g) return set_status(DPKEM_EINVAL);
  if (g->ctx) cudaSetDevice(g->ctx->device);
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  if (g->mem) {
    cudaDeviceSynchronize();
    cudaFree(g->mem);
  }
  delete g;
  return set_status(DPKEM_OK);
}

int dpkem_mixed_graph_create(dpkem_ctx *c, int form, size_t n, const dpkem_request *reqs, dpkem_graph **out) {
  if (!c || !out) return set_status(DPKEM_EINVAL);
  *out = nullptr;
  if (form != DPKEM_FORM_DP4A && form != DPKEM_FORM_TC && form != DPKEM_FORM_INT32) return set_status(DPKEM_EINVAL);
  int rc = check_requests(n, reqs);
  if (rc) return set_status(rc);
  std::lock_guard<std::mutex> lock(c->mu);
  cudaSetDevice(c->device);
  const mixed::Req *mr = reinterpret_cast<const mixed::Req *>(reqs);
  const size_t need = mixed::plan_bytes(mr, n, nullptr);
  dpkem_graph *g = new dpkem_graph();
  g->ctx = c;
  cudaError_t e = cudaMalloc(&g->mem, need);
  if (e != cudaSuccess) {
    cudaGetLastError();
    delete g;
    return set_status(DPKEM_ENOMEM);
  }
  int grid = 0;
  std::vector<uint8_t> plan(mixed::plan_struct_bytes());
  cudaStream_t cap = nullptr;
  e = persistent_grid(c, &grid);
  if (e == cudaSuccess) e = mixed::plan_build(mr, n, form, grid, g->mem, need, c->d_err, c->stream, plan.data());
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    cudaError_t le = mixed::plan_launch(plan.data(), n, grid, cap);
    e = cudaStreamEndCapture(cap, &g->graph);
    if (le != cudaSuccess) e = le;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&g->exec, g->graph, 0);
  if (cap) cudaStreamDestroy(cap);
  if (e != cudaSuccess) {
    cudaGetLastError();
    dpkem_mixed_graph_destroy(g);
    return set_status(DPKEM_ECUDA);
  }
  *out = g;
  return set_status(DPKEM_OK);
}

int dpkem_mixed_graph_launch(dpkem_graph *g, void *stream) {
  if (!g || !g->exec) return set_status(DPKEM_EINVAL);
  dpkem_ctx *c = g->ctx;
  std::lock_guard<std::mutex> lock(c->mu);
  cudaSetDevice(c->device);
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c->stream;
  cudaError_t e = cudaGraphLaunch(g->exec, st);
  if (e == cudaSuccess) e = cudaEventRecord(c->last, st);
  return set_status(cuda_status(e));
}

int dpkem_coins(dpkem_ctx *c, size_t n, size_t len, uint64_t first, const char *tag, uint8_t *out, unsigned flags,
                void *stream) {
  if (!c || !out || !tag || len == 0 || len > 136 || strlen(tag) > 16 || n > (size_t)INT32_MAX)
    return set_status(DPKEM_EINVAL);
  if (n == 0) return set_status(DPKEM_OK);
  const bool dev = (flags & DPKEM_FLAG_DEVICE_PTRS) != 0;
  std::lock_guard<std::mutex> lock(c->mu);
  cudaSetDevice(c->device);
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c->stream;
  CoinsBatch b{};
  b.len = (int)len;
  b.taglen = (int)strlen(tag);
  memcpy(b.tag, tag, b.taglen);
  cudaError_t e = cudaStreamWaitEvent(st, c->last, 0);
  if (e != cudaSuccess) return set_status(cuda_status(e));
  if (dev) {
    b.n = (int)n;
    b.first = first;
    b.out = out;
    if ((e = coins_generate(b, st)) != cudaSuccess) return set_status(cuda_status(e));
    cudaEventRecord(c->last, st);
    return set_status(DPKEM_OK);
  }
  const size_t chunk = std::max<size_t>(1, std::min(n, (c->budget / 2) / len));
  int rc = ensure_arena(c, up(chunk * len));
  if (rc) return set_status(rc);
  for (size_t f = 0; f < n; f += chunk) {
    const size_t m = std::min(chunk, n - f);
    b.n = (int)m;
    b.first = first + f;
    b.out = c->arena;
    if ((e = coins_generate(b, st)) != cudaSuccess) return set_status(cuda_status(e));
    if ((e = cudaMemcpyAsync(out + f * len, c->arena, m * len, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
      return set_status(cuda_status(e));
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return set_status(cuda_status(e));
  }
  cudaEventRecord(c->last, st);
  return set_status(DPKEM_OK);
}

int dpkem_sync(dpkem_ctx *c, void *stream) {
  if (!c) return set_status(DPKEM_EINVAL);
  std::lock_guard<std::mutex> lock(c->mu);
  cudaSetDevice(c->device);
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c->stream;
  uint32_t err = 0;
  cudaError_t e = cudaStreamSynchronize(st);
  if (e == cudaSuccess) e = cudaMemcpy(&err, c->d_err, 4, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return set_status(cuda_status(e));
  if (err) {
    cudaMemset(c->d_err, 0, 4);
    return set_status(DPKEM_ETIMEOUT);
  }
  return set_status(DPKEM_OK);
}

int dpkem_profile(dpkem_ctx *c, int enable) {
  if (!c) return set_status(DPKEM_EINVAL);
  std::lock_guard<std::mutex> lock(c->mu);
  c->profile = enable != 0;
  c->timer_stages = 0;
  return set_status(DPKEM_OK);
}

int dpkem_profile_read(dpkem_ctx *c, float *stage_ms, int max_stages) {
  if (!c || (!stage_ms && max_stages > 0)) return set_status(DPKEM_EINVAL);
  std::lock_guard<std::mutex> lock(c->mu);
  cudaSetDevice(c->device);
  const int n = c->timer_stages;
  if (n <= 0) return 0;
  if (cudaEventSynchronize(c->timer.ev[n]) != cudaSuccess) return set_status(cuda_status(cudaErrorUnknown));
  for (int k = 0; k < n && k < max_stages; k++)
    if (cudaEventElapsedTime(&stage_ms[k], c->timer.ev[k], c->timer.ev[k + 1]) != cudaSuccess)
      return set_status(cuda_status(cudaErrorUnknown));
  return n;
}

int dpkem_probe_int_peaks(dpkem_ctx *c, double *int_ops_per_s, double *keccak_per_s) {
  if (!c || !int_ops_per_s || !keccak_per_s) return set_status(DPKEM_EINVAL);
  std::lock_guard<std::mutex> lock(c->mu);
  cudaSetDevice(c->device);
  return set_status(cuda_status(probe_int_peaks(c->stream, int_ops_per_s, keccak_per_s)));
}

int dpkem_frodo_expand_a(dpkem_ctx *c, int scheme, const uint8_t *pk, uint16_t *amat, void *stream) {
  if (!c || !pk || !amat || (scheme != DPKEM_FRODO976 && scheme != DPKEM_FRODO976AES) || !aligned16(pk) ||
      !aligned16(amat))
    return set_status(DPKEM_EINVAL);
  std::lock_guard<std::mutex> lock(c->mu);
  if (cudaSetDevice(c->device) != cudaSuccess) return set_status(cuda_status(cudaErrorInvalidDevice));
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : c->stream;
  return set_status(cuda_status(frodo_expand_a(scheme == DPKEM_FRODO976AES, pk, amat, st)));
}

int dpkem_frodo_enc_shared(dpkem_ctx *c, int scheme, int form, size_t n, const uint8_t *coins, const uint8_t *pk,
                           const uint16_t *amat, uint8_t *ct, uint8_t *ss, void *stream) {
  return set_status(run_shared(c, scheme, form, OP_ENC, n, coins, pk, amat, ct, ss, stream));
}

int dpkem_frodo_dec_shared(dpkem_ctx *c, int scheme, int form, size_t n, const uint8_t *ct, const uint8_t *sk,
                           const uint16_t *amat, uint8_t *ss, void *stream) {
  return set_status(run_shared(c, scheme, form, OP_DEC, n, ct, sk, amat, ss, nullptr, stream));
}

int dpkem_keccak_f1600_lanes(dpkem_ctx *c, int lanes, size_t n, const uint64_t *in, uint64_t *out, int perms) {
  if (!c || (lanes != 1 && lanes != 2 && lanes != 5 && lanes != 25) || perms < 0 || n > (size_t)INT32_MAX)
    return set_status(DPKEM_EINVAL);
  if (n == 0) return set_status(DPKEM_OK);
  if (!in || !out || (reinterpret_cast<uintptr_t>(in) & 7) || (reinterpret_cast<uintptr_t>(out) & 7))
    return set_status(DPKEM_EINVAL);
  std::lock_guard<std::mutex> lock(c->mu);
  cudaSetDevice(c->device);
  cudaError_t e = keccak_lanes(lanes, in, out, (int)n, perms, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  return set_status(cuda_status(e));
}

int dpkem_probe_keccak_chain(dpkem_ctx *c, int lanes, int states, int perms, double *ms) {
  if (!c || !ms || (lanes != 1 && lanes != 2 && lanes != 5 && lanes != 25) || states <= 0 || perms <= 0)
    return set_status(DPKEM_EINVAL);
  std::lock_guard<std::mutex> lock(c->mu);
  cudaSetDevice(c->device);
  cudaError_t e = cudaStreamWaitEvent(c->stream, c->last, 0);
  if (e == cudaSuccess) e = probe_keccak_chain(lanes, states, perms, c->stream, ms);
  return set_status(cuda_status(e));
}

int dpkem_probe_i8_mma_peak(dpkem_ctx *c, double *macs_per_s) {
  if (!c || !macs_per_s) return set_status(DPKEM_EINVAL);
  std::lock_guard<std::mutex> lock(c->mu);
  cudaSetDevice(c->device);
  cudaError_t e = cudaStreamWaitEvent(c->stream, c->last, 0);
  if (e == cudaSuccess) e = probe_i8_mma_peak(c->stream, c->d_err, macs_per_s);
  uint32_t err = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&err, c->d_err, 4, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return set_status(cuda_status(e));
  if (err) {
    cudaMemset(c->d_err, 0, 4);
    return set_status(DPKEM_ETIMEOUT);
  }
  return set_status(DPKEM_OK);
}

int dpkem_set_tuning(const char *key, int value) {
  if (!key || value < 0) return set_status(DPKEM_EINVAL);
  Tuning &t = tuning();
  const std::string k(key);
  const bool zero_ok = k == "pipe_priority" || k == "saber_pair_max" || k == "saber_five_max" ||
                       k == "saber_finish_five_max" || k == "frodo_five_max" || k == "frodo_ss_five_max" ||
                       k == "saber_tc_ctas_per_sm" || k == "saber_warp_max" || k == "saber_finish_warp_max" ||
                       k == "frodo_warp_max" || k == "frodo_ss_warp_max" || k == "mixed_warp_max";
  if (value == 0 && !zero_ok) return set_status(DPKEM_EINVAL);
  if (k == "thread_block") {
    if (value % 32 || value > 256) return set_status(DPKEM_EINVAL);
    t.thread_block = value;
  } else if (k == "mixed_frodo_task") {
    t.mixed_frodo_task = std::min(value, 256);
  } else if (k == "mixed_pair_task") {
    t.mixed_pair_task = std::min(value, 128);
  } else if (k == "mixed_thread_task") {
    t.mixed_thread_task = std::min(value, 256);
  } else if (k == "pipe_chunks") {
    t.pipe_chunks = std::min(value, kPipeChunks);
  } else if (k == "pipe_priority") {
    t.pipe_priority = value != 0;
  } else if (k == "saber_pair_max") {
    t.saber_pair_max = value;
  } else if (k == "saber_five_max") {
    t.saber_five_max = value;
  } else if (k == "saber_finish_five_max") {
    t.saber_finish_five_max = value;
  } else if (k == "frodo_five_max") {
    t.frodo_five_max = value;
  } else if (k == "frodo_ss_five_max") {
    t.frodo_ss_five_max = value;
  } else if (k == "mixed_warp_max") {
    t.mixed_warp_max = value;
  } else if (k == "saber_warp_max") {
    t.saber_warp_max = value;
  } else if (k == "saber_finish_warp_max") {
    t.saber_finish_warp_max = value;
  } else if (k == "frodo_warp_max") {
    t.frodo_warp_max = value;
  } else if (k == "frodo_ss_warp_max") {
    t.frodo_ss_warp_max = value;
  } else if (k == "saber_tc_ctas_per_sm") {
    t.saber_tc_ctas_per_sm = std::min(value, 8);
  } else {
    return set_status(DPKEM_EINVAL);
  }
  return set_status(DPKEM_OK);
}

int dpkem_get_tuning(const char *key, int *value) {
  if (!key || !value) return set_status(DPKEM_EINVAL);
  const Tuning &t = tuning();
  const std::string k(key);
  const struct {
    const char *name;
    int v;
  } knobs[] = {{"thread_block", t.thread_block}, {"mixed_frodo_task", t.mixed_frodo_task},
               {"mixed_pair_task", t.mixed_pair_task}, {"mixed_thread_task", t.mixed_thread_task},
               {"mixed_warp_max", t.mixed_warp_max},
               {"pipe_chunks", t.pipe_chunks}, {"pipe_priority", t.pipe_priority},
               {"saber_pair_max", t.saber_pair_max}, {"saber_warp_max", t.saber_warp_max},
               {"saber_finish_warp_max", t.saber_finish_warp_max}, {"saber_five_max", t.saber_five_max},
               {"saber_finish_five_max", t.saber_finish_five_max}, {"frodo_warp_max", t.frodo_warp_max},
               {"frodo_ss_warp_max", t.frodo_ss_warp_max}, {"frodo_five_max", t.frodo_five_max},
               {"frodo_ss_five_max", t.frodo_ss_five_max}, {"saber_tc_ctas_per_sm", t.saber_tc_ctas_per_sm}};
  for (const auto &kn : knobs)
    if (k == kn.name) {
      *value = kn.v;
      return set_status(DPKEM_OK);
    }
  return set_status(DPKEM_EINVAL);
}

const char *dpkem_strerror(int s) {
  switch (s) {
    case DPKEM_OK: return "ok";
    case DPKEM_EINVAL: return "invalid argument";
    case DPKEM_ENOMEM: return "out of device memory or over the HBM budget";
    case DPKEM_ECUDA: return "CUDA runtime error";
    case DPKEM_ETIMEOUT: return "bounded device wait expired";
    case DPKEM_EUNSUPPORTED: return "unsupported form";
    case DPKEM_EAGAIN: return "nothing to take or no room yet";
    default: return "unknown status";
  }
}

int dpkem_last_status(void) { return g_last_status; }

// ---------------------------------------------------------------- compatibility shims
static std::mutex g_compat_mu;
static dpkem_ctx *g_compat = nullptr;
static size_t g_compat_batch = 768;
static int g_compat_level = 3;
static int g_compat_form = DPKEM_FORM_TC;

static dpkem_ctx *compat_ctx() {
  std::lock_guard<std::mutex> lock(g_compat_mu);
  if (!g_compat && dpkem_ctx_create(&g_compat, 0, 0) != DPKEM_OK) g_compat = nullptr;
  return g_compat;
}

void dpkem_set_compat_batch(size_t n) { g_compat_batch = n; }
void dpkem_set_compat_saber_level(int l) { g_compat_level = l; }
void dpkem_set_compat_form(int form) { g_compat_form = form; }

// The reference's mode byte (0 = DP, anything else INT32: SABER-GPU/src/cuda_kernel.cu:80,106)
// as 0 / 1, plus 2 for the tensor-core form; any other value is rejected (-1).
static int compat_form_from_mode(uint8_t mode) {
  return mode == 0 ? DPKEM_FORM_DP4A : mode == 1 ? DPKEM_FORM_INT32 : mode == 2 ? DPKEM_FORM_TC : -1;
}

void frodoKEMKeypair(uint8_t *h_pk, uint8_t *h_sk) {
  dpkem_ctx *c = compat_ctx();
  if (!c) return (void)set_status(DPKEM_ECUDA);
  std::vector<uint8_t> coins(g_compat_batch * frodo::KP_COINS);
  int rc = dpkem_coins(c, g_compat_batch, frodo::KP_COINS, 0, "kp", coins.data(), 0, nullptr);
  if (rc == DPKEM_OK)
    rc = dpkem_keypair_batch(c, DPKEM_FRODO976, g_compat_form, g_compat_batch, coins.data(), h_pk, h_sk, 0, nullptr);
  set_status(rc);
}

void frodoKEMEncap(uint8_t *ct, uint8_t *ss, const uint8_t *pk) {
  dpkem_ctx *c = compat_ctx();
  if (!c) return (void)set_status(DPKEM_ECUDA);
  std::vector<uint8_t> coins(g_compat_batch * frodo::ENC_COINS);
  int rc = dpkem_coins(c, g_compat_batch, frodo::ENC_COINS, 0, "enc", coins.data(), 0, nullptr);
  if (rc == DPKEM_OK)
    rc = dpkem_enc_batch(c, DPKEM_FRODO976, g_compat_form, g_compat_batch, coins.data(), pk, ct, ss, 0, nullptr);
  set_status(rc);
}

void frodoKEMDecap(uint8_t *ss, const uint8_t *ct, const uint8_t *sk) {
  dpkem_ctx *c = compat_ctx();
  if (!c) return (void)set_status(DPKEM_ECUDA);
  set_status(dpkem_dec_batch(c, DPKEM_FRODO976, g_compat_form, g_compat_batch, ct, sk, ss, 0, nullptr));
}

void saber_enc(uint8_t mode, uint8_t *h_k, uint8_t *h_pk, uint8_t *h_c) {
  if (compat_form_from_mode(mode) < 0) return (void)set_status(DPKEM_EINVAL);
  dpkem_ctx *c = compat_ctx();
  if (!c) return (void)set_status(DPKEM_ECUDA);
  std::vector<uint8_t> coins(g_compat_batch * 32);
  int rc = dpkem_coins(c, g_compat_batch, 32, 0, "enc", coins.data(), 0, nullptr);
  if (rc == DPKEM_OK)
    rc = dpkem_enc_batch(c, g_compat_level, compat_form_from_mode(mode), g_compat_batch, coins.data(), h_pk, h_c, h_k,
                         0, nullptr);
  set_status(rc);
}

void saber_dec(uint8_t mode, uint8_t *h_c, uint8_t *h_pk, uint8_t *h_sk, uint8_t *h_k) {
  (void)h_pk;  // the public key travels inside sk
  if (compat_form_from_mode(mode) < 0) return (void)set_status(DPKEM_EINVAL);
  dpkem_ctx *c = compat_ctx();
  if (!c) return (void)set_status(DPKEM_ECUDA);
  set_status(dpkem_dec_batch(c, g_compat_level, compat_form_from_mode(mode), g_compat_batch, h_c, h_sk, h_k, 0, nullptr));
}

}  // extern "C"
