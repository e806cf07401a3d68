// Register-resident Keccak-f[1600] for sm_100a.
//
// One thread owns one 25-lane state held as 25 x uint2 {lo, hi} (50 registers).
// Rotations are 32-bit funnel shifts (two per 64-bit lane, none for offset 0 or
// 32); theta/chi compile to LOP3.  Round constants and rho offsets are computed at
// compile time from the FIPS 202 definitions (rc(t) LFSR and the (x,y) ->
// (y, 2x+3y) walk), replacing the reference's per-thread uint64 permutation
// (FrodoKEM976-GPU/src/shake.cu:66-331, SABER-GPU/src/poly.cu:436-701) and its
// 25-lane shared-memory variant (shake.cu:380-604, poly.cu:897-1010), which ran
// without warp barriers between the steps.
#pragma once
#include <cstdint>

namespace dpkem {
namespace kc {

__host__ __device__ constexpr int rho(int i) {
  if (i == 0) return 0;
  int x = 1, y = 0;
  for (int t = 0; t < 24; t++) {
    if (x + 5 * y == i) return ((t + 1) * (t + 2) / 2) % 64;
    int nx = y, ny = (2 * x + 3 * y) % 5;
    x = nx;
    y = ny;
  }
  return -1;
}

// pi: lane (x, y) moves to (y, 2x + 3y).
__host__ __device__ constexpr int pi_dst(int i) { return (i / 5) + 5 * ((2 * (i % 5) + 3 * (i / 5)) % 5); }

__host__ __device__ constexpr uint64_t rc(int round) {
  uint32_t r = 1;
  uint64_t c = 0;
  for (int ir = 0; ir <= round; ir++) {
    c = 0;
    for (int j = 0; j < 7; j++) {
      if (r & 1) c |= 1ULL << ((1 << j) - 1);
      r = (r & 0x80) ? (((r << 1) ^ 0x71) & 0xFF) : ((r << 1) & 0xFF);
    }
  }
  return c;
}

}  // namespace kc

#define DPKEM_RC2(i) {(uint32_t)kc::rc(i), (uint32_t)(kc::rc(i) >> 32)}
__constant__ uint2 c_keccak_rc[24] = {
    DPKEM_RC2(0),  DPKEM_RC2(1),  DPKEM_RC2(2),  DPKEM_RC2(3),  DPKEM_RC2(4),  DPKEM_RC2(5),
    DPKEM_RC2(6),  DPKEM_RC2(7),  DPKEM_RC2(8),  DPKEM_RC2(9),  DPKEM_RC2(10), DPKEM_RC2(11),
    DPKEM_RC2(12), DPKEM_RC2(13), DPKEM_RC2(14), DPKEM_RC2(15), DPKEM_RC2(16), DPKEM_RC2(17),
    DPKEM_RC2(18), DPKEM_RC2(19), DPKEM_RC2(20), DPKEM_RC2(21), DPKEM_RC2(22), DPKEM_RC2(23)};
#undef DPKEM_RC2

template <int N>
__device__ __forceinline__ uint2 rotl64(uint2 v) {
  if constexpr (N == 0) {
    return v;
  } else if constexpr (N == 32) {
    return make_uint2(v.y, v.x);
  } else if constexpr (N < 32) {
    return make_uint2(__funnelshift_l(v.y, v.x, N), __funnelshift_l(v.x, v.y, N));
  } else {
    return make_uint2(__funnelshift_l(v.x, v.y, N - 32), __funnelshift_l(v.y, v.x, N - 32));
  }
}

__device__ __forceinline__ uint2 xor5(uint2 a, uint2 b, uint2 c, uint2 d, uint2 e) {
  return make_uint2(a.x ^ b.x ^ c.x ^ d.x ^ e.x, a.y ^ b.y ^ c.y ^ d.y ^ e.y);
}
// a ^ b ^ c as one LOP3.  Theta applies C[x-1] ^ rot(C[x+1], 1) to the five lanes of a
// column; written in C the compiler factors that common term out (5 XORs for D, then a
// 2-input XOR per lane: 60 ops per round where 50 three-input LOP3s suffice).  The inline
// PTX keeps each lane's update a single LOP3.
__device__ __forceinline__ uint32_t lop3_xor3(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t r;
  asm("lop3.b32 %0, %1, %2, %3, 0x96;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
  return r;
}
__device__ __forceinline__ uint2 xor3(uint2 a, uint2 b, uint2 c) {
  return make_uint2(lop3_xor3(a.x, b.x, c.x), lop3_xor3(a.y, b.y, c.y));
}
__device__ __forceinline__ uint2 chi(uint2 a, uint2 b, uint2 c) {
  return make_uint2(a.x ^ (~b.x & c.x), a.y ^ (~b.y & c.y));
}

// One round: theta, rho+pi, chi, iota.
__device__ __forceinline__ void keccak_round(uint2 (&a)[25], uint2 rcv) {
  uint2 c[5], b[25];
#pragma unroll
  for (int x = 0; x < 5; x++) c[x] = xor5(a[x], a[x + 5], a[x + 10], a[x + 15], a[x + 20]);
#pragma unroll
  for (int x = 0; x < 5; x++) {
    const uint2 r = rotl64<1>(c[(x + 1) % 5]);
    const uint2 l = c[(x + 4) % 5];
#pragma unroll
    for (int y = 0; y < 5; y++) a[x + 5 * y] = xor3(a[x + 5 * y], l, r);
  }
#define DPKEM_RHOPI(i) b[kc::pi_dst(i)] = rotl64<kc::rho(i)>(a[i]);
  DPKEM_RHOPI(0) DPKEM_RHOPI(1) DPKEM_RHOPI(2) DPKEM_RHOPI(3) DPKEM_RHOPI(4)
  DPKEM_RHOPI(5) DPKEM_RHOPI(6) DPKEM_RHOPI(7) DPKEM_RHOPI(8) DPKEM_RHOPI(9)
  DPKEM_RHOPI(10) DPKEM_RHOPI(11) DPKEM_RHOPI(12) DPKEM_RHOPI(13) DPKEM_RHOPI(14)
  DPKEM_RHOPI(15) DPKEM_RHOPI(16) DPKEM_RHOPI(17) DPKEM_RHOPI(18) DPKEM_RHOPI(19)
  DPKEM_RHOPI(20) DPKEM_RHOPI(21) DPKEM_RHOPI(22) DPKEM_RHOPI(23) DPKEM_RHOPI(24)
#undef DPKEM_RHOPI
#pragma unroll
  for (int y = 0; y < 5; y++)
#pragma unroll
    for (int x = 0; x < 5; x++) a[x + 5 * y] = chi(b[x + 5 * y], b[(x + 1) % 5 + 5 * y], b[(x + 2) % 5 + 5 * y]);
  a[0].x ^= rcv.x;
  a[0].y ^= rcv.y;
}

// Rounds per loop iteration (a tuning knob; dpcrypto_b200/tuning.json sets it at build time).
#ifndef DPKEM_KECCAK_UNROLL
#define DPKEM_KECCAK_UNROLL 2
#endif

// Rounds per loop iteration in the A-row generators' permutation: one call site per kernel,
// in a loop the compiler keeps in vector registers (a counter and a constant address
// updated per iteration), so a longer body pays there.
#ifndef DPKEM_KECCAK_UNROLL_ROWS
#define DPKEM_KECCAK_UNROLL_ROWS 1
#endif

constexpr int kKeccakUnroll = DPKEM_KECCAK_UNROLL;
constexpr int kKeccakUnrollRows = DPKEM_KECCAK_UNROLL_ROWS;

template <int U>
__device__ __forceinline__ void keccak_f1600_u(uint2 (&a)[25]) {
#pragma unroll U
  for (int r = 0; r < 24; r++) keccak_round(a, c_keccak_rc[r]);
}

__device__ __forceinline__ void keccak_f1600(uint2 (&a)[25]) { keccak_f1600_u<kKeccakUnroll>(a); }

__device__ __forceinline__ void keccak_zero(uint2 (&a)[25]) {
#pragma unroll
  for (int i = 0; i < 25; i++) a[i] = make_uint2(0u, 0u);
}

__device__ __forceinline__ uint2 ld_lane(const uint8_t *p) { return *reinterpret_cast<const uint2 *>(p); }

// Absorb `len` bytes (len % 8 == 0, p 8-byte aligned) of one message segment into a
// sponge whose current fill is `pos` bytes (a multiple of 8).  Whole rate blocks are
// absorbed with static lane indices; only the ragged head and tail use predication.
// Returns the new fill.
template <int RATE>
__device__ __forceinline__ int absorb_word(uint2 (&a)[25], int pos, uint2 w);

template <int RATE>
__device__ __forceinline__ int absorb_aligned(uint2 (&a)[25], int pos, const uint8_t *p, int len) {
  while (pos != 0 && len > 0) {
    pos = absorb_word<RATE>(a, pos, ld_lane(p));
    p += 8;
    len -= 8;
  }
  // Whole blocks: the next block's words are loaded before the permutation of this one, so
  // their global-load latency passes during the permutation instead of before the XOR.
  if (len >= RATE) {
    uint2 w[RATE / 8];
#pragma unroll
    for (int q = 0; q < RATE / 8; q++) w[q] = ld_lane(p + 8 * q);
    while (true) {
#pragma unroll
      for (int q = 0; q < RATE / 8; q++) {
        a[q].x ^= w[q].x;
        a[q].y ^= w[q].y;
      }
      p += RATE;
      len -= RATE;
      const bool more = len >= RATE;
      if (more) {
#pragma unroll
        for (int q = 0; q < RATE / 8; q++) w[q] = ld_lane(p + 8 * q);
      }
      keccak_f1600(a);
      if (!more) break;
    }
  }
  while (len > 0) {
    pos = absorb_word<RATE>(a, pos, ld_lane(p));
    p += 8;
    len -= 8;
  }
  return pos;
}

// XOR one 64-bit word into lane pos/8 (pos multiple of 8, pos < RATE); permute when full.
template <int RATE>
__device__ __forceinline__ int absorb_word(uint2 (&a)[25], int pos, uint2 w) {
#pragma unroll
  for (int q = 0; q < RATE / 8; q++)
    if (q * 8 == pos) {
      a[q].x ^= w.x;
      a[q].y ^= w.y;
    }
  pos += 8;
  if (pos == RATE) {
    keccak_f1600(a);
    pos = 0;
  }
  return pos;
}

// Apply padding (domain byte at `pos`, 0x80 in the last rate byte) and permute.
template <int RATE>
__device__ __forceinline__ void absorb_finish(uint2 (&a)[25], int pos, uint32_t domain) {
#pragma unroll
  for (int q = 0; q < RATE / 8; q++)
    if (q * 8 <= pos && pos < q * 8 + 8) {
      const int sh = 8 * (pos - q * 8);
      if (sh < 32) a[q].x ^= domain << sh;
      else a[q].y ^= domain << (sh - 32);
    }
  a[RATE / 8 - 1].y ^= 0x80000000u;
  keccak_f1600(a);
}

}  // namespace dpkem
