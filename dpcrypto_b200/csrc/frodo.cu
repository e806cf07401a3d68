// FrodoKEM-976 (SHAKE and AES variants) batched keypair / encaps / decaps: one launch per
// stage over n instances.  The stage bodies live in frodo_dev.cuh (shared with the persistent
// mixed-batch kernel); these wrappers only map blockIdx/threadIdx to instances.
#include "frodo_dev.cuh"
#include "frodo_gemm.cuh"

namespace dpkem {
namespace {

using namespace frodo;
using fdev::inst_of;

// Thread-per-instance prologues: dynamic shared memory of kParkBytes per thread parks the
// sampling stream's blocks (fdev::sample_stream).
constexpr int kParkBytes = 17 * 8;

template <int OP>
__global__ void __launch_bounds__(256) kp_prologue_kernel(FrodoBatch b) {
  extern __shared__ uint2 park[];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < b.n) fdev::kp_prologue_inst(inst_of(b, i, OP), park + threadIdx.x, blockDim.x);
}

template <int OP>
__global__ void __launch_bounds__(256) pk_hash_kernel(FrodoBatch b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < b.n) fdev::pk_hash_inst(inst_of(b, i, OP));
}

template <int MODE>
__global__ void __launch_bounds__(256) prologue_kernel(FrodoBatch b) {
  extern __shared__ uint2 park[];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < b.n) fdev::prologue_inst<MODE>(inst_of(b, i, MODE), park + threadIdx.x, blockDim.x);
}

// Decaps prologue, 64 threads = 32 instances: warp 0 runs the sampling chain, warp 1 the
// ciphertext pre-absorb of the final hash.
__global__ void __launch_bounds__(64) dec_prologue_kernel(FrodoBatch b) {
  __shared__ uint2 park[17 * 32];
  const int i = blockIdx.x * 32 + (threadIdx.x & 31);
  if (i >= b.n) return;
  if (threadIdx.x < 32) fdev::prologue_inst<OP_DEC>(inst_of(b, i, OP_DEC), park + threadIdx.x, 32);
  else fdev::ct_absorb_inst(inst_of(b, i, OP_DEC));
}

// Several lanes per state (msponge.cuh; NS = 5: five lanes, six instances per warp; NS = 1:
// a warp per instance), one warp per block.  STAGE selects the stage body: 0 keypair
// prologue, 1 H(pk), 2 encaps prologue, 3 encaps final hash, 4 decaps final hash; the
// decaps prologue below has its own kernel.
template <int STAGE, int NS>
__global__ void __launch_bounds__(32) stage_multi_kernel(FrodoBatch b) {
  using S = msp::Multi<NS>;
  __shared__ __align__(16) uint8_t xbuf[S::SMEM_PER_WARP > 0 ? S::SMEM_PER_WARP : 16];
  const S s(xbuf);
  const int g = s.state(), i = blockIdx.x * S::STATES_PER_WARP + g;
  const bool live = g < S::STATES_PER_WARP && i < b.n;
  constexpr int op = STAGE <= 1 ? OP_KEYPAIR : STAGE <= 3 ? OP_ENC : OP_DEC;
  const fdev::Inst v = inst_of(b, live ? i : b.n - 1, op);
  if constexpr (STAGE == 0) fdev::kp_prologue_multi<S>(v, s, live);
  else if constexpr (STAGE == 1) fdev::pk_hash_multi<S>(v, s, live);
  else if constexpr (STAGE == 2) fdev::prologue_multi<S, OP_ENC>(v, s, live);
  else if constexpr (STAGE == 3) fdev::ss_multi<S, OP_ENC>(v, s, live);
  else fdev::ss_multi<S, OP_DEC>(v, s, live);
}

// Decaps prologue on several lanes per state: 64 threads, warp 0 the sampling chain, warp 1
// the ciphertext pre-absorb of the final hash, for the same instances.
template <int NS>
__global__ void __launch_bounds__(64) dec_prologue_multi_kernel(FrodoBatch b) {
  using S = msp::Multi<NS>;
  __shared__ __align__(16) uint8_t xbuf[2 * (S::SMEM_PER_WARP > 0 ? S::SMEM_PER_WARP : 16)];
  const int w = threadIdx.x >> 5;
  const S s(xbuf + w * S::SMEM_PER_WARP);
  const int g = s.state(), i = blockIdx.x * S::STATES_PER_WARP + g;
  const bool live = g < S::STATES_PER_WARP && i < b.n;
  const fdev::Inst v = inst_of(b, live ? i : b.n - 1, OP_DEC);
  if (w == 0) fdev::prologue_multi<S, OP_DEC>(v, s, live);
  else fdev::ct_absorb_multi<S>(v, s, live);
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

template <int MODE, bool I32, class G>
__global__ void __launch_bounds__(256, 2) sa_dp4a_kernel(FrodoBatch b) {
  extern __shared__ __align__(1024) uint8_t smem[];
  fdev::sa_dp4a_cta<MODE, I32, G>(inst_of(b, blockIdx.x, MODE), smem);
}

template <int MODE, int NST, class G>
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
  fdev::sa_tc_cta<MODE, NST, G>(inst_of(b, blockIdx.x, MODE), smem, tbase, b.err);
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x < 32) {
    tc_fence_after();
    tmem_dealloc(tbase, fdev::TC_TMEM_COLS);
  }
}

template <bool I32, class G>
__global__ void __launch_bounds__(256, 2) kp_as_dp4a_kernel(FrodoBatch b) {
  extern __shared__ __align__(1024) uint8_t smem[];
  fdev::kp_as_dp4a_cta<I32, G>(inst_of(b, blockIdx.x, OP_KEYPAIR), smem);
}

template <int NST, class G>
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
  fdev::kp_as_tc_cta<NST, G>(inst_of(b, blockIdx.x, OP_KEYPAIR), smem, tbase, b.err);
  tc_fence_before();
  __syncthreads();
  if (threadIdx.x < 32) {
    tc_fence_after();
    tmem_dealloc(tbase, 64);
  }
}

inline int blocks_for(int n, int t) { return (n + t - 1) / t; }

// Lanes per state of a thread-level sponge stage: a warp per state up to warp_max, five lanes
// up to five_max (frodo_warp_max / frodo_five_max for the prologues, frodo_ss_warp_max /
// frodo_ss_five_max for the hashes), else one (false: the caller launches that).
template <int STAGE>
bool launch_multi(const FrodoBatch &b, int warp_max, int five_max, cudaStream_t st) {
  if (b.n <= warp_max) {
    stage_multi_kernel<STAGE, 1><<<b.n, 32, 0, st>>>(b);
    return true;
  }
  if (b.n <= five_max) {
    stage_multi_kernel<STAGE, 5><<<blocks_for(b.n, 6), 32, 0, st>>>(b);
    return true;
  }
  return false;
}

template <typename K>
cudaError_t set_smem(K kernel, int bytes) {
  return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

constexpr int kTcStages = 2;

// GT feeds the tcgen05 stage (with NST tile stages per warp), GD the dp4a / INT32 stage.
// FrodoKEM-976-AES runs its tensor stages with one tile stage: a warp spends thousands of
// cycles producing a tile, long after the previous tile's MMAs have finished, and the
// shared memory goes to the AES table copies instead.
template <int MODE, class GT, class GD, int NST>
cudaError_t launch_sa_g(const FrodoBatch &b, int form, cudaStream_t st) {
  cudaError_t e;
  if (form == FORM_TC) {
    constexpr int bytes = fdev::TcLayout<NST>::total + GT::SMEM;
    if ((e = set_smem(sa_tc_kernel<MODE, NST, GT>, bytes)) != cudaSuccess) return e;
    sa_tc_kernel<MODE, NST, GT><<<b.n, 256, bytes, st>>>(b);
  } else if (form == FORM_INT32) {
    constexpr int bytes = fdev::DP4A_SMEM + GD::SMEM;
    if ((e = set_smem(sa_dp4a_kernel<MODE, true, GD>, bytes)) != cudaSuccess) return e;
    sa_dp4a_kernel<MODE, true, GD><<<b.n, 256, bytes, st>>>(b);
  } else {
    constexpr int bytes = fdev::DP4A_SMEM + GD::SMEM;
    if ((e = set_smem(sa_dp4a_kernel<MODE, false, GD>, bytes)) != cudaSuccess) return e;
    sa_dp4a_kernel<MODE, false, GD><<<b.n, 256, bytes, st>>>(b);
  }
  return cudaGetLastError();
}

// Shared key, A in memory, tensor-core form: one GEMM over all instances (frodo_gemm.cuh).
template <int MODE>
cudaError_t launch_sa_gemm(const FrodoBatch &b, cudaStream_t st) {
  using namespace fgemm;
  cudaError_t e;
  const int groups = (b.n + INST - 1) / INST;
  tile_ab_kernel<<<blocks_for(MT * KSTEPS * 2 * 8 * 32, 256), 256, 0, st>>>(b.amat, MODE == OP_ENC ? b.pk : b.sk + LENS,
                                                                             b.abt);
  tile_s_kernel<<<blocks_for(groups * INST * NBAR * 62, 256), 256, 0, st>>>(b.rw, b.n, b.stile);
  if (MODE == OP_DEC && (e = cudaMemsetAsync(b.fail, 0, (size_t)b.n * 4, st)) != cudaSuccess) return e;
  if ((e = set_smem(gemm_kernel<MODE>, SMEM_LAUNCH)) != cudaSuccess) return e;
  const GemmArgs g{b.abt, b.stile, b.rw, MODE == OP_ENC ? b.coins : b.mu, b.ct, b.fail, b.err, b.n};
  gemm_kernel<MODE><<<MT * groups, THREADS, SMEM_LAUNCH, st>>>(g);
  return cudaGetLastError();
}

template <int MODE>
cudaError_t launch_sa(const FrodoBatch &b, int form, cudaStream_t st) {
  if (b.amat && b.abt && b.stile && form == FORM_TC) return launch_sa_gemm<MODE>(b, st);
  if (b.amat) return launch_sa_g<MODE, fdev::MemRows, fdev::MemRows, kTcStages>(b, form, st);
  if (b.aes) return launch_sa_g<MODE, fdev::AesRowsFull, fdev::AesRowsHalf, 1>(b, form, st);
  return launch_sa_g<MODE, fdev::ShakeRows, fdev::ShakeRows, kTcStages>(b, form, st);
}

// A (976 x 976 LE u16, row-major) of the public key pk, one row per thread, with the same
// row generators as the S'A stages (SHAKE128 or AES-128 rows).
template <class G>
__global__ void __launch_bounds__(256) expand_a_kernel(const uint8_t *pk, uint16_t *amat) {
  extern __shared__ __align__(16) uint8_t gmem[];
  G gen;
  gen.setup(pk, gmem);
  __syncthreads();
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  uint2 a[25];
  gen.start(a, j);
  uint2 *row = reinterpret_cast<uint2 *>(amat + (size_t)j * N);
  for (int blk = 0; blk < 12; blk++) {
    gen.next(a);
#pragma unroll
    for (int q = 0; q < 21; q++)
      if (84 * blk + 4 * q < N) row[21 * blk + q] = a[q];
  }
}

// H(pk) = SHAKE256(pk, 24) of one public key, on a warp (a warp per state).
__global__ void __launch_bounds__(32) pk_digest_kernel(const uint8_t *pk, uint8_t *out) {
  using S = msp::Multi<1>;
  const S s(nullptr);
  uint2 a[1];
  msp::zero<S>(a);
  const int pos = msp::absorb_aligned<S, 136>(a, s, 0, pk, PK, true);
  msp::absorb_finish<S, 136>(a, s, pos, 0x1Fu);
  msp::store<S>(a, s, out, 3, true);
}

template <class G, int NST>
cudaError_t launch_kp_as(const FrodoBatch &b, int form, cudaStream_t st) {
  cudaError_t e;
  if (form == FORM_TC) {
    constexpr int bytes = fdev::KptLayoutT<NST>::total + G::SMEM;
    if ((e = set_smem(kp_as_tc_kernel<NST, G>, bytes)) != cudaSuccess) return e;
    kp_as_tc_kernel<NST, G><<<b.n, 256, bytes, st>>>(b);
  } else {
    constexpr int bytes = fdev::KP_AS_SMEM + G::SMEM;
    if (form == FORM_INT32) {
      if ((e = set_smem(kp_as_dp4a_kernel<true, G>, bytes)) != cudaSuccess) return e;
      kp_as_dp4a_kernel<true, G><<<b.n, 256, bytes, st>>>(b);
    } else {
      if ((e = set_smem(kp_as_dp4a_kernel<false, G>, bytes)) != cudaSuccess) return e;
      kp_as_dp4a_kernel<false, G><<<b.n, 256, bytes, st>>>(b);
    }
  }
  return cudaGetLastError();
}

inline void mark(const FrodoBatch &b, cudaStream_t st) {
  if (b.timer) b.timer->mark(st);
}

}  // namespace

cudaError_t frodo_expand_a(int aes, const uint8_t *pk, uint16_t *amat, cudaStream_t st) {
  cudaError_t e;
  if (aes) {
    if ((e = set_smem(expand_a_kernel<fdev::AesRowsFull>, fdev::AesRowsFull::SMEM)) != cudaSuccess) return e;
    expand_a_kernel<fdev::AesRowsFull><<<blocks_for(N, 256), 256, fdev::AesRowsFull::SMEM, st>>>(pk, amat);
  } else {
    expand_a_kernel<fdev::ShakeRows><<<blocks_for(N, 256), 256, 0, st>>>(pk, amat);
  }
  return cudaGetLastError();
}

size_t frodo_gemm_ab_bytes() { return fgemm::AB_BYTES; }
size_t frodo_gemm_s_bytes(size_t n) { return fgemm::s_bytes((int)n); }

cudaError_t frodo_pk_digest(const uint8_t *pk, uint8_t *out, cudaStream_t st) {
  pk_digest_kernel<<<1, 32, 0, st>>>(pk, out);
  return cudaGetLastError();
}

cudaError_t frodo_keypair(const FrodoBatch &b, int form, cudaStream_t st) {
  if (b.n <= 0) return cudaSuccess;
  const int tb = tuning().thread_block;
  mark(b, st);
  if (!launch_multi<0>(b, tuning().frodo_warp_max, tuning().frodo_five_max, st))
    kp_prologue_kernel<OP_KEYPAIR><<<blocks_for(b.n, tb), tb, kParkBytes * tb, st>>>(b);
  mark(b, st);
  const cudaError_t e = b.aes ? launch_kp_as<fdev::AesRowsFull, 1>(b, form, st)
                             : launch_kp_as<fdev::ShakeRows, fdev::KPT_NST>(b, form, st);
  if (e != cudaSuccess) return e;
  mark(b, st);
  if (!launch_multi<1>(b, tuning().frodo_ss_warp_max, tuning().frodo_ss_five_max, st)) pk_hash_kernel<OP_KEYPAIR><<<blocks_for(b.n, tb), tb, 0, st>>>(b);
  mark(b, st);
  return cudaGetLastError();
}

cudaError_t frodo_enc(const FrodoBatch &b, int form, cudaStream_t st) {
  if (b.n <= 0) return cudaSuccess;
  const int tb = tuning().thread_block;
  mark(b, st);
  if (!launch_multi<2>(b, tuning().frodo_warp_max, tuning().frodo_five_max, st)) prologue_kernel<OP_ENC><<<blocks_for(b.n, tb), tb, kParkBytes * tb, st>>>(b);
  mark(b, st);
  cudaError_t e = launch_sa<OP_ENC>(b, form, st);
  if (e != cudaSuccess) return e;
  mark(b, st);
  if (!launch_multi<3>(b, tuning().frodo_ss_warp_max, tuning().frodo_ss_five_max, st)) ss_kernel<OP_ENC><<<blocks_for(b.n, tb), tb, 0, st>>>(b);
  mark(b, st);
  return cudaGetLastError();
}

cudaError_t frodo_dec(const FrodoBatch &b, int form, cudaStream_t st) {
  if (b.n <= 0) return cudaSuccess;
  const int tb = tuning().thread_block;
  mark(b, st);
  dec_w_kernel<<<b.n, 256, fdev::DEC_W_SMEM, st>>>(b);
  mark(b, st);
  if (b.n <= tuning().frodo_warp_max) dec_prologue_multi_kernel<1><<<b.n, 64, 0, st>>>(b);
  else if (b.n <= tuning().frodo_five_max) dec_prologue_multi_kernel<5><<<blocks_for(b.n, 6), 64, 0, st>>>(b);
  else dec_prologue_kernel<<<blocks_for(b.n, 32), 64, 0, st>>>(b);
  mark(b, st);
  cudaError_t e = launch_sa<OP_DEC>(b, form, st);
  if (e != cudaSuccess) return e;
  mark(b, st);
  if (!launch_multi<4>(b, tuning().frodo_ss_warp_max, tuning().frodo_ss_five_max, st)) ss_kernel<OP_DEC><<<blocks_for(b.n, tb), tb, 0, st>>>(b);
  mark(b, st);
  return cudaGetLastError();
}

}  // namespace dpkem
