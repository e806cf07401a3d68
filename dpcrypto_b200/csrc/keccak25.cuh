// Keccak-f[1600] with one state per warp, one 64-bit lane per thread (lanes 0..24 of the
// warp; 25..31 run along on copies of lanes 0..6 and are never stored), for sponge chains
// whose batch is too small to fill the GPU: single requests and the small batches of a
// serving loop.
//
// Thread i = x + 5y holds lane (x, y) as uint2 {lo, hi}.  One round:
//   theta  the other four lanes of column x by four shuffles, C[x] by XOR; C[x-1], C[x+1]
//          from the threads of the same row by two more
//   rho    its lane rotated by rho(x, y) (a per-thread offset: keccak5.cuh's rotv)
//   pi+chi one level of three shuffles: thread (x, y) takes the lanes that pi moves to
//          (x, y), (x+1, y) and (x+2, y) straight from their threads (the lane pi moves to
//          (x', y) comes from thread (x' + 3y mod 5) + 5x'), then chi is local
//   iota   on thread 0
// Three dependent shuffle levels (a shuffle is 26 cycles on B200, measured): 18 shuffles of
// 32-bit halves and about 21 other instructions per round, 39.5 warp instructions measured
// (ncu), against 6.2 per state on one thread per state (180 LOP3/SHF per round, 32 states per
// warp).  A warp holds one state instead of 32, so the layout pays only while the batch leaves
// warps' issue slots free; lanes per state is a tuning knob of each stage.
//
// Every lane of the warp must execute the shuffles: callers keep whole warps in step and
// predicate only global-memory accesses.
#pragma once
#include <cstdint>

#include "keccak.cuh"
#include "keccak5.cuh"

namespace dpkem {
namespace k25 {

struct Lane {
  int i;                 // lane index x + 5y this thread holds (threads 25..31: a copy of i - 25)
  int col[4];            // threads holding (x, y+1 .. y+4)
  int left, right;       // (x-1, y), (x+1, y)
  int pi[3];             // the threads whose lanes pi moves to (x, y), (x+1, y), (x+2, y)
  uint32_t rot, swap;    // rho(x, y) mod 32, all-ones when rho >= 32
  uint32_t iota;         // all-ones on thread 0
};

__device__ __forceinline__ Lane make_lane() {
  Lane k;
  const int lane = threadIdx.x & 31;
  k.i = lane < 25 ? lane : lane - 25;
  const int x = k.i % 5, y = k.i / 5;
#pragma unroll
  for (int d = 1; d < 5; d++) k.col[d - 1] = x + 5 * ((y + d) % 5);
  k.left = (x + 4) % 5 + 5 * y;
  k.right = (x + 1) % 5 + 5 * y;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    const int xp = (x + d) % 5;
    k.pi[d] = (xp + 3 * y) % 5 + 5 * xp;
  }
  int r = 0;
#pragma unroll
  for (int j = 0; j < 25; j++)
    if (j == k.i) r = kc::rho(j);
  k.rot = (uint32_t)(r & 31);
  k.swap = r >= 32 ? 0xFFFFFFFFu : 0u;
  k.iota = lane == 0 ? 0xFFFFFFFFu : 0u;
  return k;
}

__device__ __forceinline__ void round25(uint2 &v, const Lane &k, uint2 rcv) {
  const uint2 t1 = k5::shfl(v, k.col[0]), t2 = k5::shfl(v, k.col[1]), t3 = k5::shfl(v, k.col[2]),
              t4 = k5::shfl(v, k.col[3]);
  const uint2 c = xor5(v, t1, t2, t3, t4);
  const uint2 cl = k5::shfl(c, k.left), cr = rotl64<1>(k5::shfl(c, k.right));
  v = xor3(v, cl, cr);
  v = k5::rotv(v, k.rot, k.swap);
  const uint2 b = k5::shfl(v, k.pi[0]), b1 = k5::shfl(v, k.pi[1]), b2 = k5::shfl(v, k.pi[2]);
  v = chi(b, b1, b2);
  v.x ^= rcv.x & k.iota;
  v.y ^= rcv.y & k.iota;
}

__device__ __forceinline__ void f1600(uint2 &v, const Lane &k) {
#pragma unroll 4
  for (int r = 0; r < 24; r++) round25(v, k, c_keccak_rc[r]);
}

}  // namespace k25
}  // namespace dpkem
