// Integer-pipe peak probes used as roofline denominators for the Keccak-bound kernels.
//
//   int_mix:  16 independent dependency chains per thread of LOP3 (3-input XOR) and
//             SHF.L.W (funnel rotate) in Keccak's 11:5 ratio, no memory traffic; reports
//             32-bit integer ops/s over a full-occupancy grid.
//   keccak:   back-to-back Keccak-f[1600] permutations on register-resident states
//             (the same keccak_f1600 the KEM kernels use); reports permutations/s.
// Both are timed with CUDA events on the launch stream after a warm-up launch.
#include "common.cuh"
#include "keccak.cuh"

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

}  // namespace

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
