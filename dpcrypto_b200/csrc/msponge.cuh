// Sponge helpers over the multi-lane Keccak layouts, so that a stage body is written once for
// five lanes per state (keccak5.cuh, six states per warp) and a warp per state
// (keccak25.cuh, one state per warp).
//
// A layout S gives each thread S::NS slots of the state (uint2 a[S::NS]); slot y holds rate
// lane S::lane(y).  Every thread of the warp runs every call (the permutation shuffles);
// `live` predicates the global-memory accesses of a state without an instance, and
// S::writer() drops the duplicate lanes a layout keeps (the 25-lane form's threads 25..31).
#pragma once
#include <cstdint>

#include "keccak.cuh"
#include "keccak25.cuh"
#include "keccak5.cuh"

namespace dpkem {
namespace msp {

template <int NS>
struct Multi;

// Five lanes per state: thread t of group g holds lanes t, t + 5, ..., t + 20.
template <>
struct Multi<5> {
  static constexpr int NS = 5, STATES_PER_WARP = 6, SMEM_PER_WARP = k5::kSmemPerWarp;
  k5::Lanes k;
  __device__ explicit Multi(uint8_t *warp_smem) : k(k5::make_lanes(warp_smem)) {}
  __device__ int state() const { return (threadIdx.x & 31) / 5; }  // 6 for lanes 30-31 (no state)
  __device__ bool writer() const { return true; }
  __device__ int lane(int y) const { return k.t + 5 * y; }
  __device__ void perm(uint2 (&a)[5]) const { k5::f1600(a, k); }
  template <int I>
  __device__ uint2 get(const uint2 (&a)[5]) const {
    return k5::shfl(a[I / 5], k.base + I % 5);
  }
};

// A warp per state: thread i holds lane i (threads 25..31 a copy of lane i - 25).
template <>
struct Multi<1> {
  static constexpr int NS = 1, STATES_PER_WARP = 1, SMEM_PER_WARP = 0;
  k25::Lane k;
  __device__ explicit Multi(uint8_t *) : k(k25::make_lane()) {}
  __device__ int state() const { return 0; }
  __device__ bool writer() const { return (threadIdx.x & 31) < 25; }
  __device__ int lane(int) const { return k.i; }
  __device__ void perm(uint2 (&a)[1]) const { k25::f1600(a[0], k); }
  template <int I>
  __device__ uint2 get(const uint2 (&a)[1]) const {
    return k5::shfl(a[0], I);
  }
};

template <class S>
__device__ __forceinline__ void zero(uint2 (&a)[S::NS]) {
#pragma unroll
  for (int y = 0; y < S::NS; y++) a[y] = make_uint2(0u, 0u);
}

// Keep lanes 0 .. n-1, clear the rest.
template <class S>
__device__ __forceinline__ void keep(uint2 (&a)[S::NS], const S &s, int n) {
#pragma unroll
  for (int y = 0; y < S::NS; y++)
    if (s.lane(y) >= n) a[y] = make_uint2(0u, 0u);
}

// XOR w into lane I (the owner's copy of w is the one used).
template <class S, int I>
__device__ __forceinline__ void xor_lane(uint2 (&a)[S::NS], const S &s, uint2 w) {
#pragma unroll
  for (int y = 0; y < S::NS; y++)
    if (s.lane(y) == I) {
      a[y].x ^= w.x;
      a[y].y ^= w.y;
    }
}

// Lanes 0..3 of a finished state `src` moved (XORed) into lanes D..D+3 of `dst`.
template <class S, int D>
__device__ __forceinline__ void move4(uint2 (&dst)[S::NS], const uint2 (&src)[S::NS], const S &s) {
  xor_lane<S, D + 0>(dst, s, s.template get<0>(src));
  xor_lane<S, D + 1>(dst, s, s.template get<1>(src));
  xor_lane<S, D + 2>(dst, s, s.template get<2>(src));
  xor_lane<S, D + 3>(dst, s, s.template get<3>(src));
}

// Absorb whole 8-byte words (len % 8 == 0, p 8-byte aligned) at fill `pos` (a multiple of
// 8); returns the new fill.
// Whole blocks at fill 0 load the next block's words before permuting the current one, so the
// global-load latency passes during the permutation.
template <class S, int RATE>
__device__ __forceinline__ int absorb_aligned(uint2 (&a)[S::NS], const S &s, int pos, const uint8_t *p, int len,
                                              bool live) {
  constexpr int W = RATE / 8;
  if (pos == 0 && len >= RATE) {
    uint2 w[S::NS];
#pragma unroll
    for (int y = 0; y < S::NS; y++) {
      const int q = s.lane(y);
      w[y] = (q < W && live) ? ld_lane(p + 8 * q) : make_uint2(0u, 0u);
    }
    while (true) {
#pragma unroll
      for (int y = 0; y < S::NS; y++) {
        a[y].x ^= w[y].x;
        a[y].y ^= w[y].y;
      }
      p += RATE;
      len -= RATE;
      const bool more = len >= RATE;
      if (more) {
#pragma unroll
        for (int y = 0; y < S::NS; y++) {
          const int q = s.lane(y);
          if (q < W && live) w[y] = ld_lane(p + 8 * q);
        }
      }
      s.perm(a);
      if (!more) break;
    }
  }
  while (len > 0) {
    const int take = min(len, RATE - pos);
    const int q0 = pos / 8, nq = take / 8;
#pragma unroll
    for (int y = 0; y < S::NS; y++) {
      const int q = s.lane(y);
      if (q < W && q >= q0 && q < q0 + nq && live) {
        const uint2 w = ld_lane(p + 8 * (q - q0));
        a[y].x ^= w.x;
        a[y].y ^= w.y;
      }
    }
    pos += take;
    p += take;
    len -= take;
    if (pos == RATE) {
      s.perm(a);
      pos = 0;
    }
  }
  return pos;
}

// Padding (domain byte at `pos`, 0x80 in the last rate byte), then the permutation.
template <class S, int RATE>
__device__ __forceinline__ void absorb_finish(uint2 (&a)[S::NS], const S &s, int pos, uint32_t domain) {
  const int qd = pos / 8, sh = 8 * (pos % 8), ql = RATE / 8 - 1;
#pragma unroll
  for (int y = 0; y < S::NS; y++) {
    const int q = s.lane(y);
    if (q == qd) {
      if (sh < 32) a[y].x ^= domain << sh;
      else a[y].y ^= domain << (sh - 32);
    }
    if (q == ql) a[y].y ^= 0x80000000u;
  }
  s.perm(a);
}

// Squeeze `len` bytes (a multiple of 8) of a finished state to dst.
template <class S, int RATE>
__device__ __forceinline__ void squeeze(uint2 (&a)[S::NS], const S &s, uint8_t *dst, int len, bool live) {
  constexpr int W = RATE / 8;
  for (int off = 0;; off += RATE) {
#pragma unroll
    for (int y = 0; y < S::NS; y++) {
      const int q = s.lane(y);
      if (q < W && off + 8 * q < len && live && s.writer()) *reinterpret_cast<uint2 *>(dst + off + 8 * q) = a[y];
    }
    if (off + RATE >= len) break;
    s.perm(a);
  }
}

// Store lanes 0 .. nw-1 of a state to dst.
template <class S>
__device__ __forceinline__ void store(const uint2 (&a)[S::NS], const S &s, uint8_t *dst, int nw, bool live) {
#pragma unroll
  for (int y = 0; y < S::NS; y++) {
    const int q = s.lane(y);
    if (q < nw && live && s.writer()) *reinterpret_cast<uint2 *>(dst + 8 * q) = a[y];
  }
}

}  // namespace msp
}  // namespace dpkem
