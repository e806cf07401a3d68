// Seeded synthetic coins on the device: out[i] = SHAKE256(00..1F || LE64(first+i) || tag, len).
// One thread per instance; the whole message fits one SHAKE256 block and len <= 136
// bytes needs one squeeze.  This is the counter-mode stream the benchmarks and the
// compatibility shims draw keypair/encaps randomness from (the reference instead fills
// instance 0 with 0,1,2,... at FrodoKEM976-GPU/src/cuda_kernel.cu:51-53).
#include "coins_dev.cuh"
#include "common.cuh"

namespace dpkem {
namespace {

__global__ void __launch_bounds__(128) coins_kernel(CoinsBatch b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= b.n) return;
  coin_generate(default_coin_key(), b.first + (uint64_t)i, b.tag, b.taglen, b.len, b.out + (size_t)i * b.len);
}

}  // namespace

cudaError_t coins_generate(const CoinsBatch &b, cudaStream_t st) {
  if (b.n <= 0) return cudaSuccess;
  coins_kernel<<<(b.n + 127) / 128, 128, 0, st>>>(b);
  return cudaGetLastError();
}

}  // namespace dpkem
