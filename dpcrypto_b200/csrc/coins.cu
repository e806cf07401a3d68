// Seeded synthetic coins on the device: out[i] = SHAKE256(00..1F || LE64(first+i) || tag, len).
// One thread per instance; the whole message fits one SHAKE256 block and len <= 136
// bytes needs one squeeze.  This is the counter-mode stream the benchmarks and the
// compatibility shims draw keypair/encaps randomness from (the reference instead fills
// instance 0 with 0,1,2,... at FrodoKEM976-GPU/src/cuda_kernel.cu:51-53).
#include "common.cuh"
#include "keccak.cuh"

namespace dpkem {
namespace {

__global__ void __launch_bounds__(128) coins_kernel(CoinsBatch b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= b.n) return;
  uint2 a[25];
  keccak_zero(a);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const uint32_t k0 = 8 * q;  // key bytes 00 01 .. 1F
    a[q] = make_uint2(k0 | ((k0 + 1) << 8) | ((k0 + 2) << 16) | ((k0 + 3) << 24),
                      (k0 + 4) | ((k0 + 5) << 8) | ((k0 + 6) << 16) | ((k0 + 7) << 24));
  }
  const uint64_t idx = b.first + (uint64_t)i;
  a[4] = make_uint2((uint32_t)idx, (uint32_t)(idx >> 32));
  for (int t = 0; t < b.taglen; t++) {
    const int pos = 40 + t, q = pos >> 3, sh = 8 * (pos & 7);
    const uint32_t v = b.tag[t];
    if (q == 5) {
      if (sh < 32) a[5].x ^= v << sh;
      else a[5].y ^= v << (sh - 32);
    } else {
      if (sh < 32) a[6].x ^= v << sh;
      else a[6].y ^= v << (sh - 32);
    }
  }
  absorb_finish<136>(a, 40 + b.taglen, 0x1Fu);
  uint8_t *out = b.out + (size_t)i * b.len;
#pragma unroll
  for (int q = 0; q < 17; q++) {
    for (int k = 0; k < 8; k++) {
      const int pos = 8 * q + k;
      if (pos < b.len) out[pos] = (uint8_t)((k < 4 ? a[q].x >> (8 * k) : a[q].y >> (8 * (k - 4))) & 0xFFu);
    }
  }
}

}  // namespace

cudaError_t coins_generate(const CoinsBatch &b, cudaStream_t st) {
  if (b.n <= 0) return cudaSuccess;
  coins_kernel<<<(b.n + 127) / 128, 128, 0, st>>>(b);
  return cudaGetLastError();
}

}  // namespace dpkem
