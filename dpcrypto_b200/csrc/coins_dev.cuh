// Counter-mode coin stream on the device: SHAKE256(key(32) || LE64(index) || tag, len),
// len <= 136 so one absorb block and one squeeze suffice (one Keccak-f per output).
// Used by dpkem_coins (key 00 01 .. 1F) and by the persistent mixed kernel, which draws
// keypair / encaps randomness for requests that carry none.
#pragma once
#include "keccak.cuh"

namespace dpkem {

struct CoinKey {
  uint2 w[4];  // the 32-byte key as little-endian 64-bit lanes
};

__host__ __device__ inline CoinKey default_coin_key() {
  CoinKey k{};
  for (int q = 0; q < 4; q++) {
    const uint32_t k0 = 8 * q;  // bytes 00 01 .. 1F
    k.w[q] = make_uint2(k0 | ((k0 + 1) << 8) | ((k0 + 2) << 16) | ((k0 + 3) << 24),
                        (k0 + 4) | ((k0 + 5) << 8) | ((k0 + 6) << 16) | ((k0 + 7) << 24));
  }
  return k;
}

// Writes `len` coin bytes to out (8-byte stores when out is 8-aligned and len % 8 == 0).
__device__ __forceinline__ void coin_generate(const CoinKey &key, uint64_t index, const uint8_t *tag, int taglen,
                                              int len, uint8_t *out) {
  uint2 a[25];
  keccak_zero(a);
#pragma unroll
  for (int q = 0; q < 4; q++) a[q] = key.w[q];
  a[4] = make_uint2((uint32_t)index, (uint32_t)(index >> 32));
  for (int t = 0; t < taglen; t++) {  // tag bytes at message offsets 40 ..
    const int pos = 40 + t, q = pos >> 3, sh = 8 * (pos & 7);
    const uint32_t v = tag[t];
    if (q == 5) {  // constant indices keep the state in registers
      if (sh < 32) a[5].x ^= v << sh;
      else a[5].y ^= v << (sh - 32);
    } else {
      if (sh < 32) a[6].x ^= v << sh;
      else a[6].y ^= v << (sh - 32);
    }
  }
  absorb_finish<136>(a, 40 + taglen, 0x1Fu);
  if ((len & 7) == 0 && (reinterpret_cast<uintptr_t>(out) & 7) == 0) {
#pragma unroll
    for (int q = 0; q < 17; q++)
      if (8 * q < len) *reinterpret_cast<uint2 *>(out + 8 * q) = a[q];
    return;
  }
#pragma unroll
  for (int q = 0; q < 17; q++) {
    for (int k = 0; k < 8; k++) {
      const int pos = 8 * q + k;
      if (pos < len) out[pos] = (uint8_t)((k < 4 ? a[q].x >> (8 * k) : a[q].y >> (8 * (k - 4))) & 0xFFu);
    }
  }
}

}  // namespace dpkem
