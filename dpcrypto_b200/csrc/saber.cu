// Saber (LightSaber l=2, Saber l=3, FireSaber l=4) batched keypair / encaps / decaps: one
// launch per stage over n instances.  The stage bodies live in saber_dev.cuh (shared with
// the persistent mixed-batch kernel); these wrappers only map blockIdx/threadIdx to instances.
#include <algorithm>

#include "saber_dev.cuh"

namespace dpkem {
namespace {

using sdev::inst_of;
using sdev::PL;
using sdev::Scr;

// One or two lanes per state: 32 instances per block.  Warp 0 = hash chain + GenSecret XOF
// (a thread per instance); GenMatrix XOF on warp 1 (a thread per instance, PAIR = false,
// blockDim 64) or on warps 1-2 (a lane pair per instance, PAIR = true, blockDim 96).  Pairs shorten the longest chain
// while the batch leaves SM sub-partitions idle, and cost more issue slots per state once
// it does not (tuning knob saber_pair_max).
template <int L, int OP, bool PAIR>
__global__ void __launch_bounds__(96) prologue_kernel(SaberBatch b) {
  if (!PAIR || threadIdx.x < 32) {
    const int i = blockIdx.x * 32 + (threadIdx.x & 31);
    if (i < b.n) sdev::prologue_inst<L, OP>(inst_of<L>(b, i, OP), threadIdx.x >> 5);
    return;
  }
  const int t = threadIdx.x - 32, i = blockIdx.x * 32 + (t >> 1);
  const bool live = i < b.n;
  sdev::matrix_pair<L, OP>(inst_of<L>(b, live ? i : b.n - 1, OP), t & 1, live);
}

// Several lanes per state (msponge.cuh; NS = 5: five lanes, six instances per warp; NS = 1:
// a warp per instance).  Two warps per block: warp 0 the hash chain and GenSecret, warp 1
// GenMatrix, for the same instances.
template <int L, int OP, int NS>
__global__ void __launch_bounds__(64) prologue_multi_kernel(SaberBatch b) {
  using S = msp::Multi<NS>;
  __shared__ __align__(16) uint8_t xbuf[2 * (S::SMEM_PER_WARP > 0 ? S::SMEM_PER_WARP : 16)];
  const int w = threadIdx.x >> 5;
  const S s(xbuf + w * S::SMEM_PER_WARP);
  const int g = s.state(), i = blockIdx.x * S::STATES_PER_WARP + g;
  const bool live = g < S::STATES_PER_WARP && i < b.n;
  sdev::prologue_multi<S, L, OP>(inst_of<L>(b, live ? i : b.n - 1, OP), s, w, live);
}

template <int L, int OP, int NS>
void launch_prologue_multi(const SaberBatch &b, cudaStream_t st) {
  constexpr int spw = msp::Multi<NS>::STATES_PER_WARP;
  prologue_multi_kernel<L, OP, NS><<<(b.n + spw - 1) / spw, 64, 0, st>>>(b);
}

// Lanes per state of the prologue's sponges for a batch of n: a warp per state up to
// saber_warp_max, five lanes up to saber_five_max, a pair (GenMatrix only) up to
// saber_pair_max, else one.
template <int L, int OP>
void launch_prologue(const SaberBatch &b, cudaStream_t st) {
  const int pb = (b.n + 31) / 32;
  if (b.n <= tuning().saber_warp_max) launch_prologue_multi<L, OP, 1>(b, st);
  else if (b.n <= tuning().saber_five_max) launch_prologue_multi<L, OP, 5>(b, st);
  else if (b.n <= tuning().saber_pair_max) prologue_kernel<L, OP, true><<<pb, 96, 0, st>>>(b);
  else prologue_kernel<L, OP, false><<<pb, 64, 0, st>>>(b);
}

// Encaps finish on lane pairs, 64 threads = 32 instances.
template <int L>
__global__ void __launch_bounds__(64) finish_enc_pair_kernel(SaberBatch b) {
  const int t = blockIdx.x * 64 + threadIdx.x, i = t >> 1;
  const bool live = i < b.n;
  sdev::finish_enc_pair<L>(inst_of<L>(b, live ? i : b.n - 1, OP_ENC), t & 1, live);
}

// Encaps / keypair finish on several lanes per state, one warp per block.
template <int L, int OP, int NS>
__global__ void __launch_bounds__(32) finish_multi_kernel(SaberBatch b) {
  using S = msp::Multi<NS>;
  __shared__ __align__(16) uint8_t xbuf[S::SMEM_PER_WARP > 0 ? S::SMEM_PER_WARP : 16];
  const S s(xbuf);
  const int g = s.state(), i = blockIdx.x * S::STATES_PER_WARP + g;
  const bool live = g < S::STATES_PER_WARP && i < b.n;
  const sdev::Inst v = inst_of<L>(b, live ? i : b.n - 1, OP);
  if (OP == OP_ENC) sdev::finish_enc_multi<S, L>(v, s, live);
  else sdev::finish_kp_multi<S, L>(v, s, live);
}

// The finish on a warp per state or five lanes per state when n is within the thresholds;
// false otherwise.
template <int L, int OP>
bool launch_finish_multi(const SaberBatch &b, cudaStream_t st) {
  if (b.n <= tuning().saber_finish_warp_max) {
    finish_multi_kernel<L, OP, 1><<<b.n, 32, 0, st>>>(b);
    return true;
  }
  if (b.n <= tuning().saber_finish_five_max) {
    finish_multi_kernel<L, OP, 5><<<(b.n + 5) / 6, 32, 0, st>>>(b);
    return true;
  }
  return false;
}

template <int L, int OP>
__global__ void __launch_bounds__(256) finish_kernel(SaberBatch b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < b.n) sdev::finish_inst<L, OP>(inst_of<L>(b, i, OP));
}

__host__ __device__ constexpr int op_of(int mode) {
  return mode == sdev::PM_KEYPAIR ? OP_KEYPAIR : mode == sdev::PM_ENC ? OP_ENC : OP_DEC;
}

template <int L, int MODE, bool I32>
__global__ void __launch_bounds__(256) product_dp4a_kernel(SaberBatch b) {
  extern __shared__ __align__(1024) uint8_t sm[];
  sdev::product_dp4a_cta<L, MODE, I32>(inst_of<L>(b, blockIdx.x, op_of(MODE)), sm);
}

template <int L, int MODE>
__global__ void __launch_bounds__(256) product_tc_kernel(SaberBatch b) {
  using Y = PL<L>;
  extern __shared__ __align__(1024) uint8_t sm[];
  uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + Y::TSLOT);
  if (threadIdx.x < 32) {
    tmem_alloc(tslot, 32);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tslot;
  sdev::product_tc_cta<L, MODE>(inst_of<L>(b, blockIdx.x, op_of(MODE)), sm, tbase, b.err);
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x < 32) {
    tc_fence_after();
    tmem_dealloc(tbase, 32);
  }
}

// Persistent tensor-core product: each CTA keeps its TMEM columns and mbarrier across the
// instances it takes (i = blockIdx.x, + gridDim.x, ...) and loads the next instance's
// packed operands into registers while the current one is processed, so an instance's
// global-load latency hides behind the previous instance's work.  The launch bound asks
// for five resident CTAs per SM (48 registers; shared memory also allows five): the phases
// of an instance are latency-bound, so a fifth CTA's warps hide more of them (l=3 product
// stages at 4,096 instances: 0.161 ms at four CTAs of 54 registers, 0.148 ms at five).
template <int L, int MODE>
__global__ void __launch_bounds__(256, 5) product_tc_persistent_kernel(SaberBatch b) {
  using Y = PL<L>;
  extern __shared__ __align__(1024) uint8_t sm[];
  uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + Y::TSLOT);
  uint64_t *bar = reinterpret_cast<uint64_t *>(sm + Y::BAR);
  if (threadIdx.x < 32) {
    tmem_alloc(tslot, 32);
    tmem_relinquish();
  }
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tslot;
  constexpr int op = op_of(MODE);
  sdev::OperandPrefetch<L, MODE> pf;
  int i = blockIdx.x;
  if (i < b.n) pf.load(inst_of<L>(b, i, op));
  uint32_t phase = 0;
  bool ok = true;
  for (; i < b.n; i += gridDim.x) {
    pf.store(sm);  // the staging area is free: the previous instance ended with a CTA barrier
    __syncthreads();
    if (i + (int)gridDim.x < b.n) pf.load(inst_of<L>(b, i + gridDim.x, op));
    const sdev::Inst v = inst_of<L>(b, i, op);
    sdev::unpack_operands<L, MODE>(v, sm);
    __syncthreads();
    ok = sdev::tc_mma_epilogue<L, MODE>(v, sm, tbase, b.err, phase) && ok;
    phase ^= 1u;
  }
  if (threadIdx.x == 0 && ok) mbar_inval(bar);
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x < 32) {
    tc_fence_after();
    tmem_dealloc(tbase, 32);
  }
}

template <typename K>
cudaError_t prep(K kernel, int bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

template <int L, int MODE>
cudaError_t launch_product(const SaberBatch &b, int form, cudaStream_t st) {
  using Y = PL<L>;
  cudaError_t e;
  if (form == FORM_TC) {
    constexpr int bytes = Y::TC_TOTAL;
    const int per_sm = tuning().saber_tc_ctas_per_sm;
    if (per_sm > 0) {
      // persistent: per_sm CTAs per SM, several instances each.  The CTAs never wait on one
      // another, so a grid larger than what is resident only queues; TMEM (32 columns per
      // CTA) fits 16 CTAs per SM.
      static int sms = 0;  // per process and instantiation
      if (!sms) {
        if ((e = prep(product_tc_persistent_kernel<L, MODE>, bytes)) != cudaSuccess) return e;
        if ((e = cudaFuncSetAttribute(product_tc_persistent_kernel<L, MODE>,
                                      cudaFuncAttributePreferredSharedMemoryCarveout, 100)) != cudaSuccess)
          return e;
        int dev = 0, m = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&m, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        sms = m > 0 ? m : 1;
      }
      const int grid = std::min(b.n, sms * per_sm);
      product_tc_persistent_kernel<L, MODE><<<grid, 256, bytes, st>>>(b);
    } else {
      if ((e = prep(product_tc_kernel<L, MODE>, bytes)) != cudaSuccess) return e;
      product_tc_kernel<L, MODE><<<b.n, 256, bytes, st>>>(b);
    }
  } else if (form == FORM_INT32) {
    constexpr int bytes = Y::DP4A_TOTAL;
    if ((e = prep(product_dp4a_kernel<L, MODE, true>, bytes)) != cudaSuccess) return e;
    product_dp4a_kernel<L, MODE, true><<<b.n, 256, bytes, st>>>(b);
  } else {
    constexpr int bytes = Y::DP4A_TOTAL;
    if ((e = prep(product_dp4a_kernel<L, MODE, false>, bytes)) != cudaSuccess) return e;
    product_dp4a_kernel<L, MODE, false><<<b.n, 256, bytes, st>>>(b);
  }
  return cudaGetLastError();
}

inline void mark(const SaberBatch &b, cudaStream_t st) {
  if (b.timer) b.timer->mark(st);
}

template <int L>
cudaError_t run(const SaberBatch &b, int op, int form, cudaStream_t st) {
  const int tb = tuning().thread_block;
  const int fb = (b.n + tb - 1) / tb;
  cudaError_t e;
  mark(b, st);
  switch (op) {
    case OP_KEYPAIR:
      launch_prologue<L, OP_KEYPAIR>(b, st);
      mark(b, st);
      if ((e = launch_product<L, sdev::PM_KEYPAIR>(b, form, st)) != cudaSuccess) return e;
      mark(b, st);
      if (!launch_finish_multi<L, OP_KEYPAIR>(b, st)) finish_kernel<L, OP_KEYPAIR><<<fb, tb, 0, st>>>(b);
      break;
    case OP_ENC:
      launch_prologue<L, OP_ENC>(b, st);
      mark(b, st);
      if ((e = launch_product<L, sdev::PM_ENC>(b, form, st)) != cudaSuccess) return e;
      mark(b, st);
      if (!launch_finish_multi<L, OP_ENC>(b, st)) {
        if (b.n <= tuning().saber_pair_max) finish_enc_pair_kernel<L><<<(b.n + 31) / 32, 64, 0, st>>>(b);
        else finish_kernel<L, OP_ENC><<<fb, tb, 0, st>>>(b);
      }
      break;
    default:
      if ((e = launch_product<L, sdev::PM_DEC_INNER>(b, form, st)) != cudaSuccess) return e;
      mark(b, st);
      launch_prologue<L, OP_DEC>(b, st);
      mark(b, st);
      if ((e = launch_product<L, sdev::PM_DEC_CMP>(b, form, st)) != cudaSuccess) return e;
      mark(b, st);
      finish_kernel<L, OP_DEC><<<fb, tb, 0, st>>>(b);
      break;
  }
  mark(b, st);
  return cudaGetLastError();
}

cudaError_t dispatch(const SaberBatch &b, int op, int form, cudaStream_t st) {
  if (b.n <= 0) return cudaSuccess;
  switch (b.level) {
    case 2: return run<2>(b, op, form, st);
    case 3: return run<3>(b, op, form, st);
    case 4: return run<4>(b, op, form, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace

size_t saber_scratch_bytes(int level) {
  switch (level) {
    case 2: return Scr<2>::BYTES;
    case 3: return Scr<3>::BYTES;
    case 4: return Scr<4>::BYTES;
    default: return 0;
  }
}

cudaError_t saber_keypair(const SaberBatch &b, int form, cudaStream_t st) { return dispatch(b, OP_KEYPAIR, form, st); }
cudaError_t saber_enc(const SaberBatch &b, int form, cudaStream_t st) { return dispatch(b, OP_ENC, form, st); }
cudaError_t saber_dec(const SaberBatch &b, int form, cudaStream_t st) { return dispatch(b, OP_DEC, form, st); }

}  // namespace dpkem
