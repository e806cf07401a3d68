// FrodoKEM-976-SHAKE batched keypair / encaps / decaps: one launch per stage over n
// instances.  The stage bodies live in frodo_dev.cuh (shared with the persistent
// mixed-batch kernel); these wrappers only map blockIdx/threadIdx to instances.
#include "frodo_dev.cuh"

namespace dpkem {
namespace {

using namespace frodo;
using fdev::inst_of;

template <int OP>
__global__ void __launch_bounds__(256) kp_prologue_kernel(FrodoBatch b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < b.n) fdev::kp_prologue_inst(inst_of(b, i, OP));
}

template <int OP>
__global__ void __launch_bounds__(256) pk_hash_kernel(FrodoBatch b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < b.n) fdev::pk_hash_inst(inst_of(b, i, OP));
}

template <int MODE>
__global__ void __launch_bounds__(256) prologue_kernel(FrodoBatch b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < b.n) fdev::prologue_inst<MODE>(inst_of(b, i, MODE));
}

// Decaps prologue, 64 threads = 32 instances: warp 0 runs the sampling chain, warp 1 the
// ciphertext pre-absorb of the final hash.
__global__ void __launch_bounds__(64) dec_prologue_kernel(FrodoBatch b) {
  const int i = blockIdx.x * 32 + (threadIdx.x & 31);
  if (i >= b.n) return;
  if (threadIdx.x < 32) fdev::prologue_inst<OP_DEC>(inst_of(b, i, OP_DEC));
  else fdev::ct_absorb_inst(inst_of(b, i, OP_DEC));
}

template <int MODE>
__global__ void __launch_bounds__(256) ss_kernel(FrodoBatch b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < b.n) fdev::ss_inst<MODE>(inst_of(b, i, MODE));
}

__global__ void __launch_bounds__(256) dec_w_kernel(FrodoBatch b) {
  extern __shared__ __align__(1024) uint8_t smem[];
  fdev::dec_w_cta(inst_of(b, blockIdx.x, OP_DEC), smem);
}

template <int MODE, bool I32>
__global__ void __launch_bounds__(256, 2) sa_dp4a_kernel(FrodoBatch b) {
  extern __shared__ __align__(1024) uint8_t smem[];
  fdev::sa_dp4a_cta<MODE, I32>(inst_of(b, blockIdx.x, MODE), smem);
}

template <int MODE, int NST>
__global__ void __launch_bounds__(256, 2) sa_tc_kernel(FrodoBatch b) {
  using L = fdev::TcLayout<NST>;
  extern __shared__ __align__(1024) uint8_t smem[];
  uint32_t *tslot = reinterpret_cast<uint32_t *>(smem + L::tslot);
  if (threadIdx.x < 32) {
    tmem_alloc(tslot, fdev::TC_TMEM_COLS);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tslot;
  fdev::sa_tc_cta<MODE, NST>(inst_of(b, blockIdx.x, MODE), smem, tbase, b.err);
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x < 32) {
    tc_fence_after();
    tmem_dealloc(tbase, fdev::TC_TMEM_COLS);
  }
}

template <bool I32>
__global__ void __launch_bounds__(256, 2) kp_as_dp4a_kernel(FrodoBatch b) {
  extern __shared__ __align__(1024) uint8_t smem[];
  fdev::kp_as_dp4a_cta<I32>(inst_of(b, blockIdx.x, OP_KEYPAIR), smem);
}

__global__ void __launch_bounds__(256, 2) kp_as_tc_kernel(FrodoBatch b) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint32_t tslot;
  if (threadIdx.x < 32) {
    tmem_alloc(&tslot, 64);
    tmem_relinquish();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = tslot;
  fdev::kp_as_tc_cta(inst_of(b, blockIdx.x, OP_KEYPAIR), smem, tbase, b.err);
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x < 32) {
    tc_fence_after();
    tmem_dealloc(tbase, 64);
  }
}

inline int blocks_for(int n, int t) { return (n + t - 1) / t; }

template <typename K>
cudaError_t set_smem(K kernel, int bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

constexpr int kTcStages = 2;

template <int MODE>
cudaError_t launch_sa(const FrodoBatch &b, int form, cudaStream_t st) {
  cudaError_t e;
  if (form == FORM_TC) {
    constexpr int bytes = fdev::TcLayout<kTcStages>::total;
    if ((e = set_smem(sa_tc_kernel<MODE, kTcStages>, bytes)) != cudaSuccess) return e;
    sa_tc_kernel<MODE, kTcStages><<<b.n, 256, bytes, st>>>(b);
  } else if (form == FORM_INT32) {
    if ((e = set_smem(sa_dp4a_kernel<MODE, true>, fdev::DP4A_SMEM)) != cudaSuccess) return e;
    sa_dp4a_kernel<MODE, true><<<b.n, 256, fdev::DP4A_SMEM, st>>>(b);
  } else {
    if ((e = set_smem(sa_dp4a_kernel<MODE, false>, fdev::DP4A_SMEM)) != cudaSuccess) return e;
    sa_dp4a_kernel<MODE, false><<<b.n, 256, fdev::DP4A_SMEM, st>>>(b);
  }
  return cudaGetLastError();
}

inline void mark(const FrodoBatch &b, cudaStream_t st) {
  if (b.timer) b.timer->mark(st);
}

}  // namespace

cudaError_t frodo_keypair(const FrodoBatch &b, int form, cudaStream_t st) {
  if (b.n <= 0) return cudaSuccess;
  const int tb = tuning().thread_block;
  mark(b, st);
  kp_prologue_kernel<OP_KEYPAIR><<<blocks_for(b.n, tb), tb, 0, st>>>(b);
  mark(b, st);
  if (form == FORM_TC) {
    cudaError_t e = set_smem(kp_as_tc_kernel, fdev::KptLayout::total);
    if (e != cudaSuccess) return e;
    kp_as_tc_kernel<<<b.n, 256, fdev::KptLayout::total, st>>>(b);
  } else if (form == FORM_INT32) {
    kp_as_dp4a_kernel<true><<<b.n, 256, fdev::KP_AS_SMEM, st>>>(b);
  } else {
    kp_as_dp4a_kernel<false><<<b.n, 256, fdev::KP_AS_SMEM, st>>>(b);
  }
  mark(b, st);
  pk_hash_kernel<OP_KEYPAIR><<<blocks_for(b.n, tb), tb, 0, st>>>(b);
  mark(b, st);
  return cudaGetLastError();
}

cudaError_t frodo_enc(const FrodoBatch &b, int form, cudaStream_t st) {
  if (b.n <= 0) return cudaSuccess;
  const int tb = tuning().thread_block;
  mark(b, st);
  prologue_kernel<OP_ENC><<<blocks_for(b.n, tb), tb, 0, st>>>(b);
  mark(b, st);
  cudaError_t e = launch_sa<OP_ENC>(b, form, st);
  if (e != cudaSuccess) return e;
  mark(b, st);
  ss_kernel<OP_ENC><<<blocks_for(b.n, tb), tb, 0, st>>>(b);
  mark(b, st);
  return cudaGetLastError();
}

cudaError_t frodo_dec(const FrodoBatch &b, int form, cudaStream_t st) {
  if (b.n <= 0) return cudaSuccess;
  const int tb = tuning().thread_block;
  mark(b, st);
  dec_w_kernel<<<b.n, 256, fdev::DEC_W_SMEM, st>>>(b);
  mark(b, st);
  dec_prologue_kernel<<<blocks_for(b.n, 32), 64, 0, st>>>(b);
  mark(b, st);
  cudaError_t e = launch_sa<OP_DEC>(b, form, st);
  if (e != cudaSuccess) return e;
  mark(b, st);
  ss_kernel<OP_DEC><<<blocks_for(b.n, tb), tb, 0, st>>>(b);
  mark(b, st);
  return cudaGetLastError();
}

}  // namespace dpkem
