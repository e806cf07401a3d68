// Keccak-f[1600] on a lane pair, for sponges on the critical path of a latency-bound stage.
//
// Threads 2i and 2i+1 of a warp hold one state in bit-interleaved form: thread p keeps bit
// 2k + p of every 64-bit lane as bit k of a 32-bit word (25 registers).  A rotation by an
// even offset 2k is a 32-bit rotation by k on both threads; an odd offset 2k + 1 swaps the
// halves (even' = rot(odd, k + 1), odd' = rot(even, k)), one shuffle with the partner.  A
// round is 90 integer operations and 17 shuffles per thread instead of 180 operations on
// one thread.  Where a stage has one warp per SM sub-partition, a warp is bound by its own
// issue rate (the 16-lane integer pipe takes a warp instruction every two cycles), so
// halving the instructions per state shortens a sponge chain; measured on Saber's
// GenMatrix (23 permutations, 4096 instances) the chain takes 10 % less time than on one
// thread, less than the instruction count suggests because of the shuffle latency on the
// critical path of every round and the conversions of the squeezed words.
//
// Sponge bytes cross the boundary through to_slice (a 64-bit word into this thread's
// 32 bits) and from_slice (this thread's 32-bit half of the natural word: p = 0 the low
// half, p = 1 the high half).  Both are a byte permute and three delta swaps of an
// interleave / de-interleave of 32 bits.  Every thread of the warp must execute the
// shuffles: callers keep whole warps in step and predicate only memory accesses.
#pragma once
#include <cstdint>

#include "keccak.cuh"

namespace dpkem {
namespace kpair {

// Bit k of the result = bit 2k + p of w.
__host__ __device__ constexpr uint32_t slice_of(uint64_t w, int p) {
  uint32_t s = 0;
  for (int k = 0; k < 32; k++) s |= (uint32_t)((w >> (2 * k + p)) & 1u) << k;
  return s;
}

#define DPKEM_RCS(i) slice_of(kc::rc(i), 0), slice_of(kc::rc(i), 1)
__constant__ uint32_t c_rc_slice[48] = {
    DPKEM_RCS(0),  DPKEM_RCS(1),  DPKEM_RCS(2),  DPKEM_RCS(3),  DPKEM_RCS(4),  DPKEM_RCS(5),
    DPKEM_RCS(6),  DPKEM_RCS(7),  DPKEM_RCS(8),  DPKEM_RCS(9),  DPKEM_RCS(10), DPKEM_RCS(11),
    DPKEM_RCS(12), DPKEM_RCS(13), DPKEM_RCS(14), DPKEM_RCS(15), DPKEM_RCS(16), DPKEM_RCS(17),
    DPKEM_RCS(18), DPKEM_RCS(19), DPKEM_RCS(20), DPKEM_RCS(21), DPKEM_RCS(22), DPKEM_RCS(23)};
#undef DPKEM_RCS

__device__ __forceinline__ uint32_t partner(uint32_t x) { return __shfl_xor_sync(0xffffffffu, x, 1); }

// Lane rotation by R on this thread's slice; q = 1 - p.
template <int R>
__device__ __forceinline__ uint32_t rot(uint32_t own, uint32_t q) {
  if constexpr (R == 0) {
    return own;
  } else if constexpr (R % 2 == 0) {
    return __funnelshift_l(own, own, R / 2);
  } else {
    const uint32_t x = partner(own);
    return __funnelshift_l(x, x, R / 2 + q);
  }
}

__device__ __forceinline__ void round(uint32_t (&a)[25], uint32_t rc, uint32_t q) {
  uint32_t c[5], b[25];
#pragma unroll
  for (int x = 0; x < 5; x++) c[x] = a[x] ^ a[x + 5] ^ a[x + 10] ^ a[x + 15] ^ a[x + 20];
#pragma unroll
  for (int x = 0; x < 5; x++) {
    const uint32_t r = rot<1>(c[(x + 1) % 5], q), l = c[(x + 4) % 5];
#pragma unroll
    for (int y = 0; y < 5; y++) a[x + 5 * y] = lop3_xor3(a[x + 5 * y], l, r);
  }
#define DPKEM_RHOPI(i) b[kc::pi_dst(i)] = rot<kc::rho(i)>(a[i], q);
  DPKEM_RHOPI(0) DPKEM_RHOPI(1) DPKEM_RHOPI(2) DPKEM_RHOPI(3) DPKEM_RHOPI(4)
  DPKEM_RHOPI(5) DPKEM_RHOPI(6) DPKEM_RHOPI(7) DPKEM_RHOPI(8) DPKEM_RHOPI(9)
  DPKEM_RHOPI(10) DPKEM_RHOPI(11) DPKEM_RHOPI(12) DPKEM_RHOPI(13) DPKEM_RHOPI(14)
  DPKEM_RHOPI(15) DPKEM_RHOPI(16) DPKEM_RHOPI(17) DPKEM_RHOPI(18) DPKEM_RHOPI(19)
  DPKEM_RHOPI(20) DPKEM_RHOPI(21) DPKEM_RHOPI(22) DPKEM_RHOPI(23) DPKEM_RHOPI(24)
#undef DPKEM_RHOPI
#pragma unroll
  for (int y = 0; y < 5; y++)
#pragma unroll
    for (int x = 0; x < 5; x++)
      a[x + 5 * y] = b[x + 5 * y] ^ (~b[(x + 1) % 5 + 5 * y] & b[(x + 2) % 5 + 5 * y]);
  a[0] ^= rc;
}

__device__ __forceinline__ void f1600(uint32_t (&a)[25], int p) {
  const uint32_t q = 1u - (uint32_t)p;
#pragma unroll kKeccakUnroll
  for (int r = 0; r < 24; r++) {
    const uint32_t e = c_rc_slice[2 * r], o = c_rc_slice[2 * r + 1];  // warp-uniform loads
    round(a, p ? o : e, q);
  }
}

__device__ __forceinline__ void zero(uint32_t (&a)[25]) {
#pragma unroll
  for (int i = 0; i < 25; i++) a[i] = 0u;
}

// This thread's slice of the 64-bit word w = {lo, hi}: the p-bits of lo and hi are merged
// into one word (lo's at even positions, hi's at odd) and de-interleaved.
__device__ __forceinline__ uint32_t to_slice(uint2 w, int p) {
  const uint32_t lo = w.x >> p, hi = w.y << (1 - p);
  uint32_t x = (lo & 0x55555555u) | (hi & 0xAAAAAAAAu), t;
  t = (x ^ (x >> 1)) & 0x22222222u;
  x ^= t ^ (t << 1);
  t = (x ^ (x >> 2)) & 0x0C0C0C0Cu;
  x ^= t ^ (t << 2);
  t = (x ^ (x >> 4)) & 0x00F000F0u;
  x ^= t ^ (t << 4);
  return __byte_perm(x, 0, 0x3120);
}

// This thread's 32-bit half of the natural word whose slices the pair holds (p = 0: bits
// 0-31, p = 1: bits 32-63).  Shuffles with the partner: every thread of the warp calls it.
__device__ __forceinline__ uint32_t from_slice(uint32_t own, int p) {
  const uint32_t other = partner(own);
  // bytes (even0, odd0, even1, odd1) for the low half, (even2, odd2, even3, odd3) for the high
  uint32_t x = __byte_perm(own, other, p ? 0x3726u : 0x5140u), t;
  t = (x ^ (x >> 4)) & 0x00F000F0u;
  x ^= t ^ (t << 4);
  t = (x ^ (x >> 2)) & 0x0C0C0C0Cu;
  x ^= t ^ (t << 2);
  t = (x ^ (x >> 1)) & 0x22222222u;
  x ^= t ^ (t << 1);
  return x;
}

// Padding (domain byte at `pos`, 0x80 in the last rate byte) and the permutation.
template <int RATE>
__device__ __forceinline__ void absorb_finish(uint32_t (&a)[25], int pos, uint32_t domain, int p) {
  const int sh = 8 * (pos & 7);
  const uint2 w = sh < 32 ? make_uint2(domain << sh, 0u) : make_uint2(0u, domain << (sh - 32));
  const uint32_t s = to_slice(w, p);
#pragma unroll
  for (int q = 0; q < RATE / 8; q++)
    if (q == (pos >> 3)) a[q] ^= s;
  a[RATE / 8 - 1] ^= p ? 0x80000000u : 0u;  // bit 63 = odd slice, bit 31
  f1600(a, p);
}

// Absorbs `len` bytes (len % 8 == 0, 8-byte aligned) at fill `pos` (a multiple of 8);
// both threads of the pair read the same words.  Returns the new fill.
template <int RATE>
__device__ __forceinline__ int absorb_aligned(uint32_t (&a)[25], int pos, const uint8_t *m, int len, int p) {
  while (pos != 0 && len > 0) {
#pragma unroll
    for (int q = 0; q < RATE / 8; q++)
      if (q * 8 == pos) a[q] ^= to_slice(ld_lane(m), p);
    pos += 8;
    m += 8;
    len -= 8;
    if (pos == RATE) {
      f1600(a, p);
      pos = 0;
    }
  }
  // Whole blocks: the next block's words are loaded before this block's permutation, so the
  // global-load latency passes during it.
  if (len >= RATE) {
    uint2 w[RATE / 8];
#pragma unroll
    for (int q = 0; q < RATE / 8; q++) w[q] = ld_lane(m + 8 * q);
    while (true) {
#pragma unroll
      for (int q = 0; q < RATE / 8; q++) a[q] ^= to_slice(w[q], p);
      m += RATE;
      len -= RATE;
      const bool more = len >= RATE;
      if (more) {
#pragma unroll
        for (int q = 0; q < RATE / 8; q++) w[q] = ld_lane(m + 8 * q);
      }
      f1600(a, p);
      if (!more) break;
    }
  }
  while (len > 0) {
#pragma unroll
    for (int q = 0; q < RATE / 8; q++)
      if (q * 8 == pos) a[q] ^= to_slice(ld_lane(m), p);
    pos += 8;
    m += 8;
    len -= 8;
  }
  return pos;
}

// Squeezes `len` bytes (len % 8 == 0) from a finished sponge: each thread writes its 4-byte
// half of every word, the pair writes whole words; `live` = false only keeps the thread in
// step with the warp.
template <int RATE>
__device__ __forceinline__ void squeeze(uint32_t (&a)[25], uint8_t *dst, int len, int p, bool live) {
  for (int off = 0;; off += RATE) {
#pragma unroll
    for (int q = 0; q < RATE / 8; q++)
      if (off + 8 * q < len) {
        const uint32_t h = from_slice(a[q], p);
        if (live) *reinterpret_cast<uint32_t *>(dst + off + 8 * q + 4 * p) = h;
      }
    if (off + RATE >= len) break;
    f1600(a, p);
  }
}

}  // namespace kpair
}  // namespace dpkem
