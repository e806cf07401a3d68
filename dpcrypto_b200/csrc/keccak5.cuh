// Keccak-f[1600] with one state spread over five lanes of a warp, for sponge chains on the
// critical path of a latency-bound stage.
//
// A warp holds six states: lanes 5g .. 5g+4 form group g (lanes 30 and 31 run along in a
// seventh, partial group whose results are never stored).  Thread t of a group owns five of
// the 25 64-bit lanes, as uint2 {lo, hi}, in one of two layouts:
//   column layout  a[y] = lane (x = t, y)    theta's column parities are local
//   row layout     a[x] = lane (x, y = t)    chi's row neighbours are local
// One round, per thread:
//   theta  C[t] from its own five lanes; C[t-1], C[t+1] by two shuffles (as 32-bit pairs)
//   rho    its five lanes rotated by rho(t, y): a per-thread offset, so a funnel-shift pair
//          with the operands swapped by two selects when the offset is 32 or more
//   pi     column -> row layout: B[x'][y'] = A[3y' + x'][x'] after pi, so row thread y' takes
//          slot x' of column thread 3y' + x' (mod 5): five shuffles whose slot index is
//          static, only the source lane depends on the thread
//   chi    local on the row layout; iota on row thread 0, slot 0
//   back   row -> column layout through 200 bytes of shared memory per group (a transpose
//          has a thread-dependent slot on one side, which registers cannot index)
// That is 48 integer instructions, 14 shuffles and 10 shared-memory accesses per thread and
// round, against 180 integer instructions for a whole state on one thread: the dependent
// chain of a sponge gets about 2.5x fewer instructions per thread, at the price of more
// instructions per state in total.  It pays where a stage leaves SM sub-partitions idle
// (small batches, the serial sponges of a prologue) and loses where the integer pipe is
// already saturated, so lanes per state is a tuning knob of each stage.
//
// Every lane of the warp must execute the shuffles and the warp syncs: callers keep whole
// warps in step and predicate only global-memory accesses (live = false for a group without
// an instance, including the partial group of lanes 30-31).
#pragma once
#include <cstdint>

#include "keccak.cuh"

namespace dpkem {
namespace k5 {

constexpr int kGroups = 7;                      // six full groups + lanes 30-31
constexpr int kSmemPerWarp = kGroups * 25 * 8;  // transpose buffer, bytes per warp

// Per-thread constants of the layout (computed once per kernel).
struct Lanes {
  int t;         // position in the group (0..4)
  int base;      // first lane of the group
  int left;      // lane of column t - 1
  int right;     // lane of column t + 1
  int src[5];    // pi: lane of column thread 3t + x' for row slot x'
  uint32_t rot[5];   // rho(t, y) mod 32 for column slot y
  uint32_t swap[5];  // all-ones when rho(t, y) >= 32
  uint32_t iota;     // all-ones on the thread that holds lane (0, 0) in the row layout
  uint2 *xp;     // this group's transpose buffer (25 lanes) in shared memory
};

__device__ __forceinline__ Lanes make_lanes(uint8_t *warp_smem) {
  Lanes k;
  const int lane = threadIdx.x & 31;
  k.base = (lane / 5) * 5;
  k.t = lane - k.base;
  k.left = k.base + (k.t + 4) % 5;
  k.right = k.base + (k.t + 1) % 5;
#pragma unroll
  for (int x = 0; x < 5; x++) k.src[x] = k.base + (3 * k.t + x) % 5;
#pragma unroll
  for (int y = 0; y < 5; y++) {
    // kc::rho as a select chain over t (t is not a compile-time constant here)
    int r = 0;
#pragma unroll
    for (int x = 0; x < 5; x++)
      if (x == k.t) r = kc::rho(x + 5 * y);
    k.rot[y] = (uint32_t)(r & 31);
    k.swap[y] = r >= 32 ? 0xFFFFFFFFu : 0u;
  }
  k.iota = k.t == 0 ? 0xFFFFFFFFu : 0u;
  k.xp = reinterpret_cast<uint2 *>(warp_smem) + (lane / 5) * 25;
  return k;
}

__device__ __forceinline__ uint2 shfl(uint2 v, int src) {
  return make_uint2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

// 64-bit rotation by a per-thread offset: rotl(v, r) = rotl(swap(v), r - 32) for r >= 32,
// and __funnelshift_l uses the offset mod 32.
__device__ __forceinline__ uint2 rotv(uint2 v, uint32_t r, uint32_t sw) {
  const uint32_t p = (v.x & ~sw) | (v.y & sw);  // lo, or hi when swapped
  const uint32_t q = (v.y & ~sw) | (v.x & sw);
  return make_uint2(__funnelshift_l(q, p, r), __funnelshift_l(p, q, r));
}

// One round; a[] enters and leaves in the column layout.
__device__ __forceinline__ void round5(uint2 (&a)[5], const Lanes &k, uint2 rcv) {
  // theta
  const uint2 c = xor5(a[0], a[1], a[2], a[3], a[4]);
  const uint2 cl = shfl(c, k.left), cr = rotl64<1>(shfl(c, k.right));
#pragma unroll
  for (int y = 0; y < 5; y++) a[y] = xor3(a[y], cl, cr);
  // rho (column layout, lane (t, y))
#pragma unroll
  for (int y = 0; y < 5; y++) a[y] = rotv(a[y], k.rot[y], k.swap[y]);
  // pi into the row layout: slot x' of row thread t = slot x' of column thread 3t + x'
  uint2 b[5];
#pragma unroll
  for (int x = 0; x < 5; x++) b[x] = shfl(a[x], k.src[x]);
  // chi and iota (row layout, lane (x, t))
#pragma unroll
  for (int x = 0; x < 5; x++) a[x] = chi(b[x], b[(x + 1) % 5], b[(x + 2) % 5]);
  a[0].x ^= rcv.x & k.iota;
  a[0].y ^= rcv.y & k.iota;
  // back to the column layout: lane (x, t) -> buffer[5x + t] -> column thread x, slot t
#pragma unroll
  for (int x = 0; x < 5; x++) k.xp[5 * x + k.t] = a[x];
  __syncwarp();
#pragma unroll
  for (int y = 0; y < 5; y++) a[y] = k.xp[5 * k.t + y];
  // The next writes to the buffer come after the next round's theta shuffles, which every
  // lane reaches only after its reads above have returned (the shuffled value depends on
  // them), so no second warp sync is needed.
}

__device__ __forceinline__ void f1600(uint2 (&a)[5], const Lanes &k) {
#pragma unroll 1
  for (int r = 0; r < 24; r++) round5(a, k, c_keccak_rc[r]);
}

__device__ __forceinline__ void zero(uint2 (&a)[5]) {
#pragma unroll
  for (int y = 0; y < 5; y++) a[y] = make_uint2(0u, 0u);
}

// Lane i (= x + 5y) of the state, broadcast to every thread of the group.
template <int I>
__device__ __forceinline__ uint2 get(const uint2 (&a)[5], const Lanes &k) {
  return shfl(a[I / 5], k.base + I % 5);
}

// XOR w into lane I (only the owning thread's copy of w matters).
template <int I>
__device__ __forceinline__ void xor_lane(uint2 (&a)[5], const Lanes &k, uint2 w) {
  if (k.t == I % 5) {
    a[I / 5].x ^= w.x;
    a[I / 5].y ^= w.y;
  }
}

// Absorb whole 8-byte words: word q of the message block goes into lane q.  The owning
// thread loads its own words (lanes t, t + 5, ...); `len` is a multiple of 8, p 8-byte
// aligned, `pos` the current fill (multiple of 8).  Returns the new fill.
template <int RATE>
__device__ __forceinline__ int absorb_aligned(uint2 (&a)[5], const Lanes &k, int pos, const uint8_t *p, int len,
                                              bool live) {
  constexpr int W = RATE / 8;
  while (len > 0) {
    const int take = min(len, RATE - pos);
    const int q0 = pos / 8, nq = take / 8;
#pragma unroll
    for (int y = 0; y < 5; y++) {
      const int q = k.t + 5 * y;  // the lane this slot holds
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
      f1600(a, k);
      pos = 0;
    }
  }
  return pos;
}

// Padding (domain byte at `pos`, 0x80 in the last rate byte), then the permutation.
template <int RATE>
__device__ __forceinline__ void absorb_finish(uint2 (&a)[5], const Lanes &k, int pos, uint32_t domain) {
  const int qd = pos / 8, sh = 8 * (pos % 8), ql = RATE / 8 - 1;
#pragma unroll
  for (int y = 0; y < 5; y++) {
    const int q = k.t + 5 * y;
    if (q == qd) {
      if (sh < 32) a[y].x ^= domain << sh;
      else a[y].y ^= domain << (sh - 32);
    }
    if (q == ql) a[y].y ^= 0x80000000u;
  }
  f1600(a, k);
}

// Squeeze `len` bytes (a multiple of 8) to dst, permuting between rate blocks; the state
// must have been finished.  Each thread stores the lanes it owns.
template <int RATE>
__device__ __forceinline__ void squeeze(uint2 (&a)[5], const Lanes &k, uint8_t *dst, int len, bool live) {
  constexpr int W = RATE / 8;
  for (int off = 0;; off += RATE) {
#pragma unroll
    for (int y = 0; y < 5; y++) {
      const int q = k.t + 5 * y;
      if (q < W && off + 8 * q < len && live) *reinterpret_cast<uint2 *>(dst + off + 8 * q) = a[y];
    }
    if (off + RATE >= len) break;
    f1600(a, k);
  }
}

}  // namespace k5
}  // namespace dpkem
