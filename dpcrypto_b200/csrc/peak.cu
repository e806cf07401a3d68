// Integer-pipe peak probes used as roofline denominators for the Keccak-bound kernels.
//
//   int_mix:  16 independent dependency chains per thread of LOP3 (3-input XOR) and
//             SHF.L.W (funnel rotate) in Keccak's 11:5 ratio, no memory traffic; reports
//             32-bit integer ops/s over a full-occupancy grid.
//   keccak:   back-to-back Keccak-f[1600] permutations on register-resident states
//             (the same keccak_f1600 the KEM kernels use); reports permutations/s.
//   mma_i8:   one CTA per SM whose elected thread issues back-to-back 128 x 256 x 32
//             tcgen05.mma kind::i8 (u8 x s8 -> s32 in TMEM, K-major no-swizzle tiles)
//             and waits once (bounded) for their completion; reports int8 MACs/s, the
//             denominator of the products' tensor-pipe fraction.
// All are timed with CUDA events on the launch stream after a warm-up launch.
#include "common.cuh"
#include "keccak.cuh"
#include "tc.cuh"

namespace dpkem {
namespace {

__device__ __forceinline__ uint32_t lop3_xor(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t r;
  asm volatile("lop3.b32 %0, %1, %2, %3, 0x96;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
  return r;
}
__device__ __forceinline__ uint32_t shf_rot(uint32_t a, uint32_t b) {
  uint32_t r;
  asm volatile("shf.l.wrap.b32 %0, %1, %2, 13;" : "=r"(r) : "r"(a), "r"(b));
  return r;
}

__global__ void __launch_bounds__(256) int_mix_kernel(uint32_t *sink, int iters) {
  uint32_t x[16];
#pragma unroll
  for (int k = 0; k < 16; k++) x[k] = threadIdx.x * 16 + k + blockIdx.x;
  for (int it = 0; it < iters; it++) {
#pragma unroll
    for (int k = 0; k < 16; k++) {
      if (k % 16 < 11) x[k] = lop3_xor(x[k], x[(k + 5) & 15], x[(k + 11) & 15]);
      else x[k] = shf_rot(x[k], x[(k + 3) & 15]);
    }
  }
  uint32_t acc = 0;
#pragma unroll
  for (int k = 0; k < 16; k++) acc ^= x[k];
  if (acc == 0x12345678u) sink[0] = acc;
}

__global__ void __launch_bounds__(256) keccak_probe_kernel(uint32_t *sink, int perms) {
  uint2 a[25];
#pragma unroll
  for (int q = 0; q < 25; q++) a[q] = make_uint2(threadIdx.x + q, blockIdx.x ^ q);
  for (int p = 0; p < perms; p++) keccak_f1600(a);
  uint32_t acc = 0;
#pragma unroll
  for (int q = 0; q < 25; q++) acc ^= a[q].x ^ a[q].y;
  if (acc == 0x12345678u) sink[0] = acc;
}

constexpr int kProbeM = 128, kProbeN = 256, kProbeK = 32;
constexpr int kProbeSmem = (kProbeM + kProbeN) * kProbeK;  // A 4 KB | B 8 KB

__global__ void __launch_bounds__(128) mma_i8_probe_kernel(int iters, uint32_t *err) {
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint32_t tslot;
  __shared__ __align__(8) uint64_t bar;
  const int tid = threadIdx.x;
  for (int i = tid; i < kProbeSmem / 16; i += blockDim.x)
    reinterpret_cast<uint4 *>(smem)[i] = make_uint4(0x01010101u * (uint32_t)(i & 7), 0x02020202u, 0u, 0x7F7F7F7Fu);
  if (tid < 32) {
    tmem_alloc(&tslot, kProbeN);
    tmem_relinquish();
  }
  if (tid == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = tslot;
  bool ok = true;
  if (tid == 0) {
    // K-major canonical tiles: byte (row, k) at (row / 8) * 256 + (k / 16) * 128 + (row % 8) * 16 + k % 16
    const uint32_t a = smem_u32(smem), b = a + kProbeM * kProbeK;
    const uint64_t ad = sdesc(a, 128, 256), bd = sdesc(b, 128, 256);
    constexpr uint32_t id = idesc_i8(kProbeM, kProbeN, false, true, false, false);
    for (int i = 0; i < iters; i++) mma_i8(tbase, ad, bd, id, i > 0 ? 1u : 0u);
    mma_commit(&bar);
    ok = mbar_wait(&bar, 0);
    if (!ok) atomicOr(err, DEV_ERR_TIMEOUT);
    else mbar_inval(&bar);
  }
  tc_fence_before();
  __syncthreads();
  if (tid < 32) {
    tc_fence_after();
    tmem_dealloc(tbase, kProbeN);
  }
}

}  // namespace

cudaError_t probe_i8_mma_peak(cudaStream_t st, uint32_t *err, double *macs_per_s) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  const int iters = 8192;
  mma_i8_probe_kernel<<<sms, 128, kProbeSmem, st>>>(64, err);
  cudaEventRecord(t0, st);
  mma_i8_probe_kernel<<<sms, 128, kProbeSmem, st>>>(iters, err);
  cudaEventRecord(t1, st);
  cudaError_t e = cudaEventSynchronize(t1);
  float ms = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
  if (e == cudaSuccess) *macs_per_s = (double)sms * iters * kProbeM * kProbeN * kProbeK / (ms * 1e-3);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  return e == cudaSuccess ? cudaGetLastError() : e;
}

cudaError_t probe_int_peaks(cudaStream_t st, double *int_ops_per_s, double *keccak_per_s) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  uint32_t *sink = nullptr;
  cudaError_t e = cudaMalloc(&sink, 4);
  if (e != cudaSuccess) return e;
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  const int threads = 256;
  int occ_mix = 1, occ_k = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_mix, int_mix_kernel, threads, 0);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_k, keccak_probe_kernel, threads, 0);
  int blocks = sms * occ_mix;  // exactly one full wave
  float ms = 0.f;
  const int iters = 4096;
  int_mix_kernel<<<blocks, threads, 0, st>>>(sink, 64);
  cudaEventRecord(t0, st);
  int_mix_kernel<<<blocks, threads, 0, st>>>(sink, iters);
  cudaEventRecord(t1, st);
  cudaEventSynchronize(t1);
  cudaEventElapsedTime(&ms, t0, t1);
  *int_ops_per_s = (double)blocks * threads * iters * 16 / (ms * 1e-3);
  const int perms = 256;
  blocks = sms * occ_k;
  keccak_probe_kernel<<<blocks, threads, 0, st>>>(sink, 2);
  cudaEventRecord(t0, st);
  keccak_probe_kernel<<<blocks, threads, 0, st>>>(sink, perms);
  cudaEventRecord(t1, st);
  cudaEventSynchronize(t1);
  cudaEventElapsedTime(&ms, t0, t1);
  *keccak_per_s = (double)blocks * threads * perms / (ms * 1e-3);
  cudaEventDestroy(t0);
  cudaEventDestroy(t1);
  cudaFree(sink);
  return cudaGetLastError();
}

}  // namespace dpkem
