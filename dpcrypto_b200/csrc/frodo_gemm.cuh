// FrodoKEM S'A + E' and S'B + E'' + encode(mu) for a batch under one key, as one int8
// tcgen05 GEMM.
//
// With the key shared, A (976 x 976) and B (976 x 8) are the same for every instance, so
// the products of all instances are one matrix product: rows n = 8 i + k (instance i, row k
// of its S'), columns m = 0..975 for B' and 976..983 for V, D[m][n] = sum_j [A | B][j][m] S'[n][j].
// A and B are u16: their low and high bytes are two u8 limb planes, each multiplied into its
// own s32 accumulator (S' is a small signed value, exact in s8), and D = lo + 256 hi mod 2^16,
// which is all FrodoKEM-976 keeps (q = 2^16).
//
// Tiles: M = 128 columns of [A | B], N = 128 rows (16 instances), K = 32 rows of A per MMA,
// 31 K steps (976 padded to 992).  Both operands are prepared once in the exact shared-memory
// layout of one K step, so a CTA moves them with one-dimensional bulk copies (no tensor map):
//   [A | B] tile (per M tile, K step, limb, 4,096 B, MN-major, no swizzle):
//       byte (m, j) at (m / 16) * 512 + (j / 8) * 128 + (j % 8) * 16 + m % 16
//   S' tile (per 16-instance group, K step, 4,096 B, K-major, no swizzle):
//       byte (n, j) at (n / 8) * 256 + (j / 16) * 128 + (n % 8) * 16 + j % 16
// The [A | B] tiles (1,015,808 B per limb) come from the expanded matrix and the public key
// (tile_ab_kernel); the S' tiles from the sampled words of each instance (tile_s_kernel).
//
// CTA (192 threads): warp 0 lane 0 issues the bulk copies of a 6-stage ring, warp 1 lane 0 the
// MMAs (two per K step, one per limb), warps 2-5 handle the epilogue.  While the MMAs run
// they load the tile's terms into shared memory with 16-byte loads (E', or E'' + encode(mu)
// for V's columns; decaps: the expected product ct - term), then read the accumulators back
// (warp w reads TMEM lanes 32 (w % 4) .. +31, the columns m its lanes own), and either write
// the sums into the same buffer and store the ciphertext rows with 16-byte stores (encaps)
// or compare (decaps: an OR of the differences into each instance's fail word, zeroed
// before the launch).  Every wait is a bounded mbarrier wait; an expired one sets the error
// word and the CTA skips the rest.
#pragma once
#include <cstdint>

#include "frodo_dev.cuh"
#include "tc.cuh"

namespace dpkem {
namespace fgemm {

using namespace frodo;

constexpr int KSTEPS = 31;                 // 992 / 32
constexpr int MT = 8;                      // M tiles of 128 columns: [A | B] has 984
constexpr int CHUNK = 4096;                // one operand tile of one K step
constexpr int INST = 16;                   // instances per N tile
constexpr int NST = 6;                     // ring stages
constexpr int STAGE = 3 * CHUNK;           // A lo, A hi, S'
constexpr int BARS = NST * STAGE;          // full[NST], empty[NST], done
constexpr int TSLOT = BARS + (2 * NST + 1) * 8;
// Epilogue terms of the tile, [128 rows n][128 columns m] u16 (32 KB): encaps the term to add
// (E', or E'' + encode(mu) in the 8 columns of V), decaps the expected product (ct - that term).
constexpr int EBUF = (TSLOT + 16 + 127) & ~127;
constexpr int SMEM = EBUF + 128 * 128 * 2;
// Requested per CTA: more than the layout needs, so that at most two CTAs share an SM and
// their TMEM allocations (256 columns each) always fit.
constexpr int SMEM_LAUNCH = 110 * 1024;
static_assert(SMEM <= SMEM_LAUNCH, "layout exceeds the requested shared memory");
constexpr int THREADS = 192;
constexpr int TMEM_COLS = 256;             // lo accumulators 0..127, hi 128..255
constexpr size_t AB_BYTES = (size_t)MT * KSTEPS * 2 * CHUNK;
__host__ __device__ constexpr size_t s_bytes(int n) { return (size_t)((n + INST - 1) / INST) * KSTEPS * CHUNK; }

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// 16 bytes global -> shared, asynchronous (L2 only); completion by cp_async_wait_all.
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_all;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// One thread per (M tile, K step, limb, 16-column group, row j % 8): 16 bytes of a tile.
// Source: A[j][m] (u16, row-major, 976 x 976) for m < 976, B[j][m - 976] (BE16 in the public
// key after its 16-byte seed) for m < 984, zero above and for j >= 976.
__global__ void __launch_bounds__(256) tile_ab_kernel(const uint16_t *amat, const uint8_t *pk, uint8_t *ab) {
  const int t = blockIdx.x * 256 + threadIdx.x;
  if (t >= MT * KSTEPS * 2 * 8 * 32) return;
  const int jr = t & 31, mg = (t >> 5) & 7, limb = (t >> 8) & 1, ks = (t >> 9) % KSTEPS, mt = (t >> 9) / KSTEPS;
  const int j = 32 * ks + jr, m0 = 128 * mt + 16 * mg;
  uint32_t w[4] = {0u, 0u, 0u, 0u};
  if (j < N) {
#pragma unroll
    for (int q = 0; q < 16; q++) {
      const int m = m0 + q;
      uint32_t v = 0;
      if (m < N) v = amat[(size_t)j * N + m];
      else if (m < N + NBAR) v = ((uint32_t)pk[SEEDA + 2 * (NBAR * j + m - N)] << 8) | pk[SEEDA + 2 * (NBAR * j + m - N) + 1];
      w[q >> 2] |= ((limb ? v >> 8 : v) & 0xFFu) << (8 * (q & 3));
    }
  }
  uint8_t *dst = ab + ((size_t)(mt * KSTEPS + ks) * 2 + limb) * CHUNK + mg * 512 + (jr >> 3) * 128 + (jr & 7) * 16;
  *reinterpret_cast<uint4 *>(dst) = make_uint4(w[0], w[1], w[2], w[3]);
}

// One thread per (instance slot, row k, 16-column group of j): 16 s8 values of S' (the low
// bytes of the sampled words rw[i][k N + j]), zero for j >= 976 and slots past n.
__global__ void __launch_bounds__(256) tile_s_kernel(const uint16_t *rw, int n, uint8_t *st) {
  const int t = blockIdx.x * 256 + threadIdx.x;
  const int groups = (n + INST - 1) / INST;
  if (t >= groups * INST * NBAR * 62) return;
  const int g = t % 62, k = (t / 62) & 7, slot = t / (62 * NBAR);  // slot = instance
  const int j = 16 * g;
  uint4 o = make_uint4(0, 0, 0, 0);
  if (slot < n && j < N) {
    const uint16_t *src = rw + (size_t)slot * RW + k * N + j;  // 16-byte aligned: 2 (k N + 16 g)
    const uint4 x0 = *reinterpret_cast<const uint4 *>(src), x1 = *reinterpret_cast<const uint4 *>(src + 8);
    o = make_uint4(prmt(x0.x, x0.y, 0x6420), prmt(x0.z, x0.w, 0x6420), prmt(x1.x, x1.y, 0x6420),
                   prmt(x1.z, x1.w, 0x6420));
  }
  const int grp = slot / INST, n_in = 8 * (slot % INST) + k;
  uint8_t *dst = st + ((size_t)grp * KSTEPS + (j >> 5)) * CHUNK + (n_in >> 3) * 256 + ((j >> 4) & 1) * 128 + (n_in & 7) * 16;
  *reinterpret_cast<uint4 *>(dst) = o;
}

struct GemmArgs {
  const uint8_t *ab, *st;
  const uint16_t *rw;  // per instance RW words: S' | E' | E''
  const uint8_t *mu;   // encaps: coins (mu, 24 B per instance); decaps: the decoded mu'
  uint8_t *ct;         // CT bytes per instance
  uint32_t *fail;      // decaps
  uint32_t *err;
  int n;
};

template <int MODE>
__global__ void __launch_bounds__(THREADS, 1) gemm_kernel(GemmArgs g) {
  extern __shared__ __align__(1024) uint8_t sm[];
  uint64_t *full = reinterpret_cast<uint64_t *>(sm + BARS), *empty = full + NST, *done = full + 2 * NST;
  uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + TSLOT);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int mt = blockIdx.x % MT, grp = blockIdx.x / MT;
  if (warp == 0) {
    tmem_alloc(tslot, TMEM_COLS);
    tmem_relinquish();
  }
  if (tid == 32) {
    for (int s = 0; s < 2 * NST + 1; s++) mbar_init(&full[s], 1);
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tbase = *tslot;
  bool ok = true;
  if (warp == 0) {
    if (lane == 0) {  // producer
      const uint8_t *a = g.ab + (size_t)mt * KSTEPS * 2 * CHUNK, *s = g.st + (size_t)grp * KSTEPS * CHUNK;
      for (int ks = 0; ks < KSTEPS && ok; ks++) {
        const int q = ks % NST;
        if (ks >= NST) ok = mbar_wait(&empty[q], ((ks / NST) - 1) & 1);
        if (!ok) break;
        const uint32_t dst = smem_u32(sm + q * STAGE);
        mbar_expect_tx(&full[q], STAGE);
        bulk_g2s(dst, a + (size_t)ks * 2 * CHUNK, 2 * CHUNK, &full[q]);
        bulk_g2s(dst + 2 * CHUNK, s + (size_t)ks * CHUNK, CHUNK, &full[q]);
      }
      // the last commits on each stage: observed before the CTA's barriers go away
      for (int q = 0; q < NST && ok; q++) {
        const int last = KSTEPS - 1 - ((KSTEPS - 1 - q) % NST);  // last K step that used stage q
        ok = mbar_wait(&empty[q], (last / NST) & 1);
      }
      if (!ok) atomicOr(g.err, DEV_ERR_TIMEOUT);
    }
  } else if (warp == 1) {
    if (lane == 0) {  // MMA issuer
      constexpr uint32_t idesc = idesc_i8(128, 128, false, true, true, false);
      for (int ks = 0; ks < KSTEPS && ok; ks++) {
        const int q = ks % NST;
        ok = mbar_wait(&full[q], (ks / NST) & 1);
        if (!ok) break;
        tc_fence_after();
        const uint32_t base = smem_u32(sm + q * STAGE);
        const uint64_t bdesc = sdesc(base + 2 * CHUNK, 128, 256);
        mma_i8(tbase, sdesc(base, 128, 512), bdesc, idesc, ks > 0 ? 1u : 0u);
        mma_i8(tbase + 128, sdesc(base + CHUNK, 128, 512), bdesc, idesc, ks > 0 ? 1u : 0u);
        mma_commit(&empty[q]);
      }
      if (ok) mma_commit(done);
      else atomicOr(g.err, DEV_ERR_TIMEOUT);
    }
  } else {  // epilogue: warps 2..5 (128 threads), TMEM lanes 32 (warp % 4) ..
    const int et = tid - 64, lg = warp & 3, ml = 32 * lg + lane;
    uint16_t *eb = reinterpret_cast<uint16_t *>(sm + EBUF);
    // While the MMAs run: the tile's terms, row n = 8 slot + k, columns m - 128 mt.  E' rows by
    // asynchronous 16-byte copies (8 columns each); V's 8 columns (tile MT - 1, columns 80..87)
    // E'' + encode(mu), one row per thread; zeros for padding columns and absent instances.
    for (int x = et; x < 128 * 16; x += 128) {
      const int n = x >> 4, q = x & 15, i = grp * INST + (n >> 3), k = n & 7, m0 = 128 * mt + 8 * q;
      uint16_t *dst = eb + n * 128 + 8 * q;
      if (i < g.n && m0 < N) cp_async16(dst, g.rw + (size_t)i * RW + N * NBAR + k * N + m0);
      else if (!(i < g.n && m0 == N)) *reinterpret_cast<uint4 *>(dst) = make_uint4(0, 0, 0, 0);
    }
    if (mt == MT - 1) {
      const int n = et, i = grp * INST + (n >> 3), k = n & 7;
      if (i < g.n) {
        const uint4 v = *reinterpret_cast<const uint4 *>(g.rw + (size_t)i * RW + 2 * N * NBAR + k * NBAR);
        const uint8_t *mu = g.mu + (size_t)i * 24 + 3 * k;
        const uint32_t t3 = mu[0] | ((uint32_t)mu[1] << 8) | ((uint32_t)mu[2] << 16);
        const uint32_t w[4] = {v.x, v.y, v.z, v.w};
        uint32_t o[4];
#pragma unroll
        for (int h = 0; h < 4; h++) {
          const uint32_t e0 = (w[h] + (((t3 >> (6 * h)) & 7u) << 13)) & 0xFFFFu;
          const uint32_t e1 = ((w[h] >> 16) + (((t3 >> (6 * h + 3)) & 7u) << 13)) & 0xFFFFu;
          o[h] = e0 | (e1 << 16);
        }
        *reinterpret_cast<uint4 *>(eb + n * 128 + (N - 128 * mt)) = make_uint4(o[0], o[1], o[2], o[3]);
      }
    }
    // Decaps: this thread's pieces of the ciphertext tile (the compare pass below), loaded
    // now so that they arrive while the MMAs run.
    uint4 cv[INST];
    if (MODE == OP_DEC) {
#pragma unroll
      for (int sl = 0; sl < INST; sl++) {
        const int x = et + 128 * sl, n = x >> 4, q = x & 15, i = grp * INST + sl, k = n & 7, m0 = 128 * mt + 8 * q;
        cv[sl] = make_uint4(0, 0, 0, 0);
        if (i < g.n && m0 < N + NBAR)
          cv[sl] = *reinterpret_cast<const uint4 *>(g.ct + (size_t)i * CT +
                                                     (m0 < N ? 2 * (k * N + m0) : PKB + 2 * k * NBAR));
      }
    }
    cp_async_wait_all();
    asm volatile("bar.sync 1, 128;" ::: "memory");  // every epilogue warp's terms are in place
    ok = __all_sync(0xffffffffu, mbar_wait(done, 0));  // warp-uniform: tcgen05.ld is warp-wide
    if (!ok && lane == 0) atomicOr(g.err, DEV_ERR_TIMEOUT);
    tc_fence_after();
    // D + term (mod 2^16) over the terms: big-endian bytes (encaps, ready to store) or the value
    if (ok) {
#pragma unroll 1
      for (int c0 = 0; c0 < 128; c0 += 16) {
        uint32_t lo[16], hi[16];
        tmem_ld16(tbase + ((uint32_t)(32 * lg) << 16) + c0, lo);
        tmem_ld16(tbase + ((uint32_t)(32 * lg) << 16) + 128 + c0, hi);
        tmem_wait_ld();
#pragma unroll
        for (int q = 0; q < 16; q++) {
          uint16_t *e = eb + (c0 + q) * 128 + ml;
          const uint32_t x = (lo[q] + (hi[q] << 8) + (uint32_t)*e) & 0xFFFFu;
          *e = MODE == OP_ENC ? (uint16_t)((x >> 8) | (x << 8)) : (uint16_t)x;
        }
      }
    }
    asm volatile("bar.sync 1, 128;" ::: "memory");
    // Rows in 16-byte pieces: iteration s covers instance slot s (8 rows x 16 pieces = 128).
    if (ok) {
#pragma unroll
      for (int sl = 0; sl < INST; sl++) {
        const int x = et + 128 * sl, n = x >> 4, q = x & 15, i = grp * INST + sl, k = n & 7, m0 = 128 * mt + 8 * q;
        const bool live = i < g.n && m0 < N + NBAR;
        const uint4 v = *reinterpret_cast<const uint4 *>(eb + n * 128 + 8 * q);
        if (MODE == OP_ENC) {
          if (live)
            *reinterpret_cast<uint4 *>(g.ct + (size_t)i * CT + (m0 < N ? 2 * (k * N + m0) : PKB + 2 * k * NBAR)) = v;
        } else {
          // ct is big-endian: swap each 16-bit half before comparing; rows m >= 984 and
          // absent instances hold zeros on both sides
          const uint32_t d = (__byte_perm(cv[sl].x, 0, 0x2301) ^ v.x) | (__byte_perm(cv[sl].y, 0, 0x2301) ^ v.y) |
                             (__byte_perm(cv[sl].z, 0, 0x2301) ^ v.z) | (__byte_perm(cv[sl].w, 0, 0x2301) ^ v.w);
          if (__ballot_sync(0xffffffffu, live && d != 0) && lane == 0 && i < g.n) atomicOr(g.fail + i, 1u);
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    tmem_dealloc(tbase, TMEM_COLS);
  }
}

}  // namespace fgemm
}  // namespace dpkem
