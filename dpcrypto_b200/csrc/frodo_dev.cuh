// FrodoKEM-976 device routines (SHAKE and AES variants: they differ only in the A-row
// generator, see ShakeRows / AesRows), written per instance so that the batched kernels
// (frodo.cu) and the persistent mixed-batch kernel (mixed.cu) run the same code.
//
// Stages per operation (all instances independent):
//   keypair: kp_prologue (thread: seedA, 0x5F stream -> S^T,E)  ->  kp_as_dp4a (CTA: A rows
//            generated in registers, B = A S + E)  ->  pk_hash (thread: H(pk) into sk)
//   encaps:  prologue (thread: pkh, G2 = SHAKE256(pkh||mu), 0x96 stream -> S',E',E'')
//            -> sa_{dp4a,tc} (CTA: B' = S'A + E' with A never leaving the SM, V = S'B + E'',
//               C = V + Encode(mu), ct written)  ->  ss (thread: SHAKE256(ct||k))
//   decaps:  dec_w (CTA: W = C - B'S, mu' = Decode(W)) -> prologue -> sa_{dp4a,tc} in compare
//            mode -> ss with the implicit-reject select.
//
// Replaces the reference's ~20-35 launches per operation
// (FrodoKEM976-GPU/src/cuda_kernel.cu:21-335) whose A matrix made a 1.9 MB HBM round trip
// per instance (shake128_ser, shake.cu:619-644; DoDP4Av5s, matrix_kernel.cu:183-241).
#pragma once
#include "common.cuh"
#include "keccak.cuh"
#include "msponge.cuh"
#include "tc.cuh"

namespace dpkem {
namespace fdev {

using namespace frodo;

// Pointers of one instance, already offset into the caller's arrays and the scratch arena.
struct Inst {
  const uint8_t *coins;  // keypair 64 B = s||seedSE||z; enc 24 B = mu
  uint8_t *pk, *sk, *ct, *ss;
  uint16_t *rw;          // RW sampled words
  uint8_t *kk, *mu;      // 24 B each
  uint32_t *fail;
  uint2 *hs;             // 25 lanes: SHAKE256 state after ct's full blocks (decaps)
  const uint16_t *amat;  // A expanded in memory (shared-key batches), or null
  const uint8_t *pkh;    // H(pk) precomputed (shared-key encaps), or null
};

__device__ __forceinline__ Inst inst_of(const FrodoBatch &b, int i, int op) {
  Inst v;
  v.coins = b.coins ? b.coins + (size_t)i * (op == OP_KEYPAIR ? KP_COINS : ENC_COINS) : nullptr;
  const size_t ik = b.shared ? 0 : (size_t)i;  // shared-key batches: one pk / sk for all
  v.pk = b.pk ? b.pk + ik * PK : nullptr;
  v.sk = b.sk ? b.sk + ik * SK : nullptr;
  v.ct = b.ct ? b.ct + (size_t)i * CT : nullptr;
  v.ss = b.ss ? b.ss + (size_t)i * SS : nullptr;
  v.rw = b.rw + (size_t)i * RW;
  v.kk = b.kk + (size_t)i * LENSE;
  v.mu = b.mu + (size_t)i * LENMU;
  v.fail = b.fail + i;
  v.hs = b.hs ? b.hs + (size_t)i * 25 : nullptr;
  v.amat = b.amat;
  v.pkh = b.pkh;
  return v;
}

__device__ __forceinline__ uint32_t sample16(uint32_t v) {
  // Constant-time CDF sampler (FrodoKEM976-GPU/src/sample_pack.cu:13-46, table params.h:24-25).
  constexpr uint32_t cdf[10] = {5638, 15915, 23689, 28571, 31116, 32217, 32613, 32731, 32760, 32766};
  const uint32_t t = (v & 0xFFFFu) >> 1, sign = v & 1u;
  uint32_t s = 0;
#pragma unroll
  for (int c = 0; c < 10; c++) s += (cdf[c] - t) >> 31;
  return (((0u - sign) ^ s) + sign) & 0xFFFFu;
}

// The same sampler written as multiply-adds: x = CDF[c] - t by mad.lo (t * (2^32 - 1) + CDF[c])
// and s += x >> 31 by mad.hi (hi32(x * 2)), multipliers moved into registers.  The compiler
// still sees the constants: in the thread-per-instance prologue ncu shows the FMA pipe 0.4 %
// active, so these run as integer-ALU ops.  Multipliers read from constant memory do keep
// them on the FMA pipe, and that form made the prologues slower (encaps 2.10 -> 2.50 ms,
// decaps 1.50 -> 1.76 ms at 8,192), so this one stays.  Bit-identical to sample16 (checked
// exhaustively on the GPU).
struct FmaConsts {
  uint32_t neg1, two;
};
__device__ __forceinline__ FmaConsts fma_consts() {
  FmaConsts k;
  asm volatile("mov.u32 %0, 0xFFFFFFFF;" : "=r"(k.neg1));
  asm volatile("mov.u32 %0, 2;" : "=r"(k.two));
  return k;
}

__device__ __forceinline__ uint32_t sample16_fma(uint32_t v, FmaConsts k) {
  constexpr uint32_t cdf[10] = {5638, 15915, 23689, 28571, 31116, 32217, 32613, 32731, 32760, 32766};
  const uint32_t t = (v & 0xFFFFu) >> 1, sign = v & 1u;
  uint32_t s = 0;
#pragma unroll
  for (int c = 0; c < 10; c++) {
    uint32_t x;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(x) : "r"(t), "r"(k.neg1), "r"(cdf[c]));
    asm("mad.hi.u32 %0, %1, %2, %0;" : "+r"(s) : "r"(x), "r"(k.two));
  }
  return (((0u - sign) ^ s) + sign) & 0xFFFFu;
}

__device__ __forceinline__ uint2 sample_lane(uint2 w) {
  const FmaConsts k = fma_consts();
  return make_uint2(sample16_fma(w.x, k) | (sample16_fma(w.x >> 16, k) << 16),
                    sample16_fma(w.y, k) | (sample16_fma(w.y >> 16, k) << 16));
}

// Message lanes of 0x5F/0x96 || seed (24 bytes), i.e. the 25-byte sampling-stream input.
__device__ __forceinline__ void seed_stream_init(uint2 (&a)[25], uint32_t dom, uint2 s0, uint2 s1, uint2 s2) {
  keccak_zero(a);
  const uint64_t x0 = ((uint64_t)s0.y << 32) | s0.x, x1 = ((uint64_t)s1.y << 32) | s1.x,
                 x2 = ((uint64_t)s2.y << 32) | s2.x;
  const uint64_t l0 = dom | (x0 << 8), l1 = (x0 >> 56) | (x1 << 8), l2 = (x1 >> 56) | (x2 << 8), l3 = x2 >> 56;
  a[0] = make_uint2((uint32_t)l0, (uint32_t)(l0 >> 32));
  a[1] = make_uint2((uint32_t)l1, (uint32_t)(l1 >> 32));
  a[2] = make_uint2((uint32_t)l2, (uint32_t)(l2 >> 32));
  a[3] = make_uint2((uint32_t)l3, 0u);
  absorb_finish<136>(a, 25, 0x1Fu);
}

// Sample one squeezed lane (four 16-bit values) to dst[at..at+3] if at < words, and to
// dst_le too while at < le_words.  The stores are predicated, not branched around.
__device__ __forceinline__ void sample_store(uint2 w, int at, uint16_t *dst, int words, uint8_t *dst_le,
                                             int le_words) {
  const uint2 v = sample_lane(w);
  if (at < words) *reinterpret_cast<uint2 *>(dst + at) = v;
  if (dst_le && at < le_words) *reinterpret_cast<uint2 *>(dst_le + 2 * at) = v;
}

// Squeeze `words` sampled 16-bit values of the stream into dst (8-byte aligned);
// when dst_le is non-null the first `le_words` values are also written there (sk's S^T).
// With `park` (this thread's column of 17 uint2 in shared memory, `stride` apart), every block
// but the last is parked there and sampled during the permutation that produces the next one,
// one lane per round for the first 17 rounds: the CDF comparisons (FMA pipe) and the stores
// then issue between the round's ALU ops.  A thread-per-instance prologue runs about one warp
// per SM sub-partition, where the ALU pipe bounds the permutation and issue slots are free;
// sampled after the permutation instead, a block cost about 40 % more than its permutation.
__device__ __forceinline__ void sample_stream(uint2 (&a)[25], uint16_t *dst, int words, uint8_t *dst_le,
                                              int le_words, uint2 *park = nullptr, int stride = 0) {
  const int nblk = (words + 67) / 68;
  if (park != nullptr) {
    for (int blk = 0; blk + 1 < nblk; blk++) {
#pragma unroll
      for (int q = 0; q < 17; q++) park[q * stride] = a[q];
#pragma unroll 1
      for (int r = 0; r < 17; r++) {
        keccak_round(a, c_keccak_rc[r]);
        sample_store(park[r * stride], blk * 68 + 4 * r, dst, words, dst_le, le_words);
      }
#pragma unroll 1
      for (int r = 17; r < 24; r++) keccak_round(a, c_keccak_rc[r]);
    }
#pragma unroll
    for (int q = 0; q < 17; q++) sample_store(a[q], (nblk - 1) * 68 + 4 * q, dst, words, dst_le, le_words);
    return;
  }
  for (int blk = 0; blk < nblk; blk++) {
    if (blk) keccak_f1600(a);
#pragma unroll
    for (int q = 0; q < 17; q++) {
      const int w = blk * 68 + 4 * q;
      if (w < words) {
        const uint2 v = sample_lane(a[q]);
        *reinterpret_cast<uint2 *>(dst + w) = v;
        if (dst_le && w < le_words) *reinterpret_cast<uint2 *>(dst_le + 2 * w) = v;
      }
    }
  }
}

// ---------------------------------------------------------------- thread-level stages
__device__ __forceinline__ void kp_prologue_inst(const Inst &v, uint2 *park = nullptr, int stride = 0) {
  uint2 a[25];
  // seedA = SHAKE256(z, 16)
  keccak_zero(a);
  a[0] = ld_lane(v.coins + 48);
  a[1] = ld_lane(v.coins + 56);
  absorb_finish<136>(a, 16, 0x1Fu);
  *reinterpret_cast<uint2 *>(v.pk) = a[0];
  *reinterpret_cast<uint2 *>(v.pk + 8) = a[1];
  *reinterpret_cast<uint2 *>(v.sk + LENS) = a[0];
  *reinterpret_cast<uint2 *>(v.sk + LENS + 8) = a[1];
#pragma unroll
  for (int q = 0; q < 3; q++) *reinterpret_cast<uint2 *>(v.sk + 8 * q) = ld_lane(v.coins + 8 * q);
  // S^T || E = sample(SHAKE256(0x5F || seedSE))
  seed_stream_init(a, 0x5Fu, ld_lane(v.coins + 24), ld_lane(v.coins + 32), ld_lane(v.coins + 40));
  sample_stream(a, v.rw, 2 * N * NBAR, v.sk + SK_S, N * NBAR, park, stride);
}

// H(pk) = SHAKE256(pk, 24) into sk.
__device__ __forceinline__ void pk_hash_inst(const Inst &v) {
  uint2 a[25];
  keccak_zero(a);
  const int pos = absorb_aligned<136>(a, 0, v.pk, PK);
  absorb_finish<136>(a, pos, 0x1Fu);
#pragma unroll
  for (int q = 0; q < 3; q++) *reinterpret_cast<uint2 *>(v.sk + SK_PKH + 8 * q) = a[q];
}

// park / stride: shared memory for sample_stream's overlapped form (null: sample after each
// permutation, as the stages of the persistent kernels do).
template <int MODE>
__device__ __forceinline__ void prologue_inst(const Inst &v, uint2 *park = nullptr, int stride = 0) {
  uint2 a[25], pkh[3], mu[3];
  if (MODE == OP_ENC) {
    if (v.pkh) {  // shared-key batch: H(pk) hashed once
#pragma unroll
      for (int q = 0; q < 3; q++) a[q] = ld_lane(v.pkh + 8 * q);
    } else {
      keccak_zero(a);
      const int pos = absorb_aligned<136>(a, 0, v.pk, PK);
      absorb_finish<136>(a, pos, 0x1Fu);
    }
#pragma unroll
    for (int q = 0; q < 3; q++) {
      pkh[q] = a[q];
      mu[q] = ld_lane(v.coins + 8 * q);
    }
  } else {
#pragma unroll
    for (int q = 0; q < 3; q++) {
      pkh[q] = ld_lane(v.sk + SK_PKH + 8 * q);
      mu[q] = ld_lane(v.mu + 8 * q);
    }
  }
  // G2 = SHAKE256(pkh || mu, 48) = seedSE || k
  keccak_zero(a);
#pragma unroll
  for (int q = 0; q < 3; q++) {
    a[q] = pkh[q];
    a[3 + q] = mu[q];
  }
  absorb_finish<136>(a, 48, 0x1Fu);
#pragma unroll
  for (int q = 0; q < 3; q++) *reinterpret_cast<uint2 *>(v.kk + 8 * q) = a[3 + q];
  seed_stream_init(a, 0x96u, a[0], a[1], a[2]);
  sample_stream(a, v.rw, RW, nullptr, 0, park, stride);
}

// Decaps: ss = SHAKE256(ct || k-hat) absorbs the input ciphertext's 115 full rate blocks
// before k-hat is known, so that part runs beside the prologue (second role of its stage);
// the state is parked in scratch and ss_inst<OP_DEC> finishes with one permutation.
constexpr int CT_FULL = (CT / 136) * 136;  // 15,640

__device__ __forceinline__ void ct_absorb_inst(const Inst &v) {
  uint2 a[25];
  keccak_zero(a);
  absorb_aligned<136>(a, 0, v.ct, CT_FULL);
#pragma unroll
  for (int q = 0; q < 25; q++) v.hs[q] = a[q];
}

// ss = SHAKE256(ct || k); decaps selects k' or s in constant time (util.cu:193-226).
template <int MODE>
__device__ __forceinline__ void ss_inst(const Inst &v) {
  uint2 kh[3];
  if (MODE == OP_ENC) {
#pragma unroll
    for (int q = 0; q < 3; q++) kh[q] = ld_lane(v.kk + 8 * q);
  } else {
    const uint32_t m = 0u - (uint32_t)(*v.fail != 0u);
#pragma unroll
    for (int q = 0; q < 3; q++) {
      const uint2 x = ld_lane(v.kk + 8 * q), y = ld_lane(v.sk + 8 * q);
      kh[q] = make_uint2((x.x & ~m) | (y.x & m), (x.y & ~m) | (y.y & m));
    }
  }
  uint2 a[25];
  int pos;
  if (MODE == OP_DEC) {
#pragma unroll
    for (int q = 0; q < 25; q++) a[q] = v.hs[q];
    pos = absorb_aligned<136>(a, 0, v.ct + CT_FULL, CT - CT_FULL);
  } else {
    keccak_zero(a);
    pos = absorb_aligned<136>(a, 0, v.ct, CT);
  }
#pragma unroll
  for (int q = 0; q < 3; q++) pos = absorb_word<136>(a, pos, kh[q]);
  absorb_finish<136>(a, pos, 0x1Fu);
#pragma unroll
  for (int q = 0; q < 3; q++) *reinterpret_cast<uint2 *>(v.ss + 8 * q) = a[q];
}

// ---------------------------------------------------------------- several lanes per state
// The thread-level stages above with each sponge spread over several lanes (msponge.cuh:
// S = msp::Multi<5>, five lanes per state, or msp::Multi<1>, a warp per state); they write
// the same bytes.  live = false keeps a state without an instance in step (its reads stay
// in bounds, its writes are skipped).

__device__ __forceinline__ uint64_t u64_of(uint2 v) { return ((uint64_t)v.y << 32) | v.x; }
__device__ __forceinline__ uint2 uint2_of(uint64_t v) { return make_uint2((uint32_t)v, (uint32_t)(v >> 32)); }

// dom || seed (25 bytes) absorbed and finished, the 24-byte seed in lanes 0..2 of g:
// message lane j = (seed lane j-1 >> 56) | (seed lane j << 8), lane 0 with dom.
template <class S>
__device__ __forceinline__ void seed_stream_init_multi(uint2 (&a)[S::NS], const S &s, uint32_t dom,
                                                       const uint2 (&g)[S::NS]) {
  const uint64_t x0 = u64_of(s.template get<0>(g)), x1 = u64_of(s.template get<1>(g)),
                 x2 = u64_of(s.template get<2>(g));
  msp::zero<S>(a);
#pragma unroll
  for (int y = 0; y < S::NS; y++) {
    const int q = s.lane(y);
    const uint64_t l = q == 0 ? (uint64_t)dom | (x0 << 8)
                     : q == 1 ? (x0 >> 56) | (x1 << 8)
                     : q == 2 ? (x1 >> 56) | (x2 << 8)
                     : q == 3 ? (x2 >> 56)
                              : 0ull;
    a[y] = uint2_of(l);
  }
  msp::absorb_finish<S, 136>(a, s, 25, 0x1Fu);
}

// sample_stream on several lanes: each thread samples and stores the rate lanes it owns.
template <class S>
__device__ __forceinline__ void sample_stream_multi(uint2 (&a)[S::NS], const S &s, uint16_t *dst, int words,
                                                    uint8_t *dst_le, int le_words, bool live) {
  const int nblk = (words + 67) / 68;
  for (int blk = 0; blk < nblk; blk++) {
    if (blk) s.perm(a);
#pragma unroll
    for (int y = 0; y < S::NS; y++) {
      const int q = s.lane(y), w = blk * 68 + 4 * q;
      if (q < 17 && w < words && live && s.writer()) {
        const uint2 v = sample_lane(a[y]);
        *reinterpret_cast<uint2 *>(dst + w) = v;
        if (dst_le && w < le_words) *reinterpret_cast<uint2 *>(dst_le + 2 * w) = v;
      }
    }
  }
}

template <class S>
__device__ __forceinline__ void kp_prologue_multi(const Inst &v, const S &s, bool live) {
  uint2 a[S::NS], g[S::NS];
  // seedA = SHAKE256(z, 16)
  msp::zero<S>(a);
  msp::absorb_aligned<S, 136>(a, s, 0, v.coins + 48, 16, live);
  msp::absorb_finish<S, 136>(a, s, 16, 0x1Fu);
  msp::store<S>(a, s, v.pk, 2, live);
  msp::store<S>(a, s, v.sk + LENS, 2, live);
  const int q = s.lane(0);
  if (live && s.writer() && q < 3) *reinterpret_cast<uint2 *>(v.sk + 8 * q) = ld_lane(v.coins + 8 * q);
  // S^T || E = sample(SHAKE256(0x5F || seedSE))
  msp::zero<S>(g);
  msp::absorb_aligned<S, 136>(g, s, 0, v.coins + 24, 24, live);
  seed_stream_init_multi<S>(a, s, 0x5Fu, g);
  sample_stream_multi<S>(a, s, v.rw, 2 * N * NBAR, v.sk + SK_S, N * NBAR, live);
}

template <class S>
__device__ __forceinline__ void pk_hash_multi(const Inst &v, const S &s, bool live) {
  uint2 a[S::NS];
  msp::zero<S>(a);
  const int pos = msp::absorb_aligned<S, 136>(a, s, 0, v.pk, PK, live);
  msp::absorb_finish<S, 136>(a, s, pos, 0x1Fu);
  msp::store<S>(a, s, v.sk + SK_PKH, 3, live);
}

template <class S, int MODE>
__device__ __forceinline__ void prologue_multi(const Inst &v, const S &s, bool live) {
  uint2 a[S::NS], g[S::NS];
  msp::zero<S>(g);
  if (MODE == OP_ENC) {
    if (v.pkh) {  // shared-key batch: H(pk) hashed once
      msp::absorb_aligned<S, 136>(g, s, 0, v.pkh, 24, live);
    } else {
      msp::zero<S>(a);
      const int pos = msp::absorb_aligned<S, 136>(a, s, 0, v.pk, PK, live);
      msp::absorb_finish<S, 136>(a, s, pos, 0x1Fu);
#pragma unroll
      for (int y = 0; y < S::NS; y++)
        if (s.lane(y) < 3) g[y] = a[y];  // pkh = lanes 0..2
    }
    msp::absorb_aligned<S, 136>(g, s, 24, v.coins, 24, live);
  } else {
    msp::absorb_aligned<S, 136>(g, s, 0, v.sk + SK_PKH, 24, live);
    msp::absorb_aligned<S, 136>(g, s, 24, v.mu, 24, live);
  }
  // G2 = SHAKE256(pkh || mu, 48) = seedSE (lanes 0..2) || k (lanes 3..5)
  msp::absorb_finish<S, 136>(g, s, 48, 0x1Fu);
#pragma unroll
  for (int y = 0; y < S::NS; y++) {
    const int q = s.lane(y);
    if (q >= 3 && q < 6 && live && s.writer()) *reinterpret_cast<uint2 *>(v.kk + 8 * (q - 3)) = g[y];
  }
  seed_stream_init_multi<S>(a, s, 0x96u, g);
  sample_stream_multi<S>(a, s, v.rw, RW, nullptr, 0, live);
}

template <class S>
__device__ __forceinline__ void ct_absorb_multi(const Inst &v, const S &s, bool live) {
  uint2 a[S::NS];
  msp::zero<S>(a);
  msp::absorb_aligned<S, 136>(a, s, 0, v.ct, CT_FULL, live);
#pragma unroll
  for (int y = 0; y < S::NS; y++)
    if (live && s.writer()) v.hs[s.lane(y)] = a[y];
}

template <class S, int MODE>
__device__ __forceinline__ void ss_multi(const Inst &v, const S &s, bool live) {
  uint2 a[S::NS];
  int pos;
  if (MODE == OP_DEC) {
#pragma unroll
    for (int y = 0; y < S::NS; y++) a[y] = live ? v.hs[s.lane(y)] : make_uint2(0u, 0u);
    pos = msp::absorb_aligned<S, 136>(a, s, 0, v.ct + CT_FULL, CT - CT_FULL, live);
  } else {
    msp::zero<S>(a);
    pos = msp::absorb_aligned<S, 136>(a, s, 0, v.ct, CT, live);
  }
  // k (encaps) or k' / s selected in constant time (decaps), in lanes pos/8 .. pos/8 + 2
  static_assert(CT % 136 % 8 == 0 && CT % 136 + 24 < 136, "k-hat fits after ct in the last rate block");
  const uint32_t m = (MODE == OP_DEC && live) ? 0u - (uint32_t)(*v.fail != 0u) : 0u;
  const int q0 = pos / 8;
#pragma unroll
  for (int y = 0; y < S::NS; y++) {
    const int q = s.lane(y);
    if (q >= q0 && q < q0 + 3 && live) {
      uint2 x = ld_lane(v.kk + 8 * (q - q0));
      if (MODE == OP_DEC) {
        const uint2 sv = ld_lane(v.sk + 8 * (q - q0));
        x = make_uint2((x.x & ~m) | (sv.x & m), (x.y & ~m) | (sv.y & m));
      }
      a[y].x ^= x.x;
      a[y].y ^= x.y;
    }
  }
  msp::absorb_finish<S, 136>(a, s, pos + 24, 0x1Fu);
  msp::store<S>(a, s, v.ss, 3, live);
}

// ---------------------------------------------------------------- CTA-level stages (256 threads)
constexpr int DEC_W_SMEM = 2 * PKB + 4 * 64 * 4 + 64 * 2;

// decaps: W = C - B'S, mu' = Decode(W).
__device__ __forceinline__ void dec_w_cta(const Inst &v, uint8_t *smem) {
  uint16_t *bp = reinterpret_cast<uint16_t *>(smem);
  uint16_t *st = reinterpret_cast<uint16_t *>(smem + PKB);
  uint32_t(*red)[64] = reinterpret_cast<uint32_t(*)[64]>(smem + 2 * PKB);
  uint16_t *w = reinterpret_cast<uint16_t *>(smem + 2 * PKB + 4 * 64 * 4);
  const int tid = threadIdx.x;
  const uint8_t *ct = v.ct, *sk = v.sk + SK_S;
  for (int q = tid; q < PKB / 16; q += 256) {
    const uint4 x = *reinterpret_cast<const uint4 *>(ct + 16 * q);  // 8 big-endian words
    *reinterpret_cast<uint4 *>(bp + 8 * q) =
        make_uint4(prmt(x.x, 0, 0x2301), prmt(x.y, 0, 0x2301), prmt(x.z, 0, 0x2301), prmt(x.w, 0, 0x2301));
  }
  for (int q = tid; q < PKB / 8; q += 256) *reinterpret_cast<uint2 *>(st + 4 * q) = ld_lane(sk + 8 * q);
  __syncthreads();
  const int o = tid & 63, q = tid >> 6, k = o >> 3, l = o & 7;
  uint32_t acc = 0;
  for (int j = 244 * q; j < 244 * q + 244; j++) acc += (uint32_t)bp[k * N + j] * st[l * N + j];
  red[q][o] = acc;
  __syncthreads();
  if (tid < 64) {
    const uint32_t c = ((uint32_t)ct[PKB + 2 * tid] << 8) | ct[PKB + 2 * tid + 1];
    w[tid] = (uint16_t)(c - (red[0][tid] + red[1][tid] + red[2][tid] + red[3][tid]));
  }
  __syncthreads();
  if (tid < NBAR) {  // Decode row tid: 8 x 3 bits (encode_decode.cu:31-53)
    uint32_t t = 0;
#pragma unroll
    for (int c = 0; c < NBAR; c++) t |= ((((uint32_t)w[tid * NBAR + c] + (1u << 12)) >> 13) & 7u) << (3 * c);
    v.mu[3 * tid] = (uint8_t)t;
    v.mu[3 * tid + 1] = (uint8_t)(t >> 8);
    v.mu[3 * tid + 2] = (uint8_t)(t >> 16);
  }
  __syncthreads();
}

// Row j of A: state after absorbing LE16(j) || seedA with SHAKE128 padding.
__device__ __forceinline__ void row_init(uint2 (&a)[25], uint32_t j, uint2 sa0, uint2 sa1) {
  keccak_zero(a);
  a[0] = make_uint2(j | (sa0.x << 16), (sa0.x >> 16) | (sa0.y << 16));
  a[1] = make_uint2((sa0.y >> 16) | (sa1.x << 16), (sa1.x >> 16) | (sa1.y << 16));
  a[2] = make_uint2((sa1.y >> 16) | (0x1Fu << 16), 0u);
  a[20].y = 0x80000000u;
}

__device__ __forceinline__ uint32_t bswap16x2(uint32_t v0, uint32_t v1) { return prmt(v0, v1, 0x4501); }

// ---------------------------------------------------------------- A-row generators
// The stages that consume A take its rows from a generator: start(a, j) begins row j and
// every next(a) leaves the row's next 84 entries in a[0..20] (4 x u16 per lane, LE), the
// block one SHAKE128 squeeze yields.  setup() runs on all threads of the CTA before the
// CTA's first __syncthreads; `mem` is the generator's SMEM bytes of shared memory.
//   ShakeRows  FrodoKEM-976-SHAKE: row j = SHAKE128(LE16(j) || seedA), one Keccak-f per block.
//   AesRows    FrodoKEM-976-AES: A[j][8c .. 8c+7] = AES128(seedA, LE16(j) || LE16(8c) || 0^12)
//              as LE u16; a block is 10.5 AES blocks, the odd half carried to the next call.
struct ShakeRows {
  static constexpr int SMEM = 0;
  uint2 sa0, sa1;
  __device__ __forceinline__ void setup(const uint8_t *seed, uint8_t *) {
    sa0 = ld_lane(seed);
    sa1 = ld_lane(seed + 8);
  }
  __device__ __forceinline__ void start(uint2 (&a)[25], uint32_t j) { row_init(a, j, sa0, sa1); }
  __device__ __forceinline__ void next(uint2 (&a)[25]) { keccak_f1600_u<kKeccakUnrollRows>(a); }
};

// MemRows: rows of an A expanded once in memory (976 x 976 LE u16, row-major; shared-key
// batches, where every instance's A is the same).  setup() receives A's address in place of
// the seed.  Entries past column 975 of the last block are zero; padding rows (j >= 976)
// read row 975, and their secret words are zero, so they add nothing.
struct MemRows {
  static constexpr int SMEM = 0;
  const uint2 *base, *row;
  int col;
  __device__ __forceinline__ void setup(const uint8_t *amat, uint8_t *) { base = reinterpret_cast<const uint2 *>(amat); }
  __device__ __forceinline__ void start(uint2 (&)[25], uint32_t j) {
    row = base + (size_t)(j < (uint32_t)N ? j : N - 1) * (N / 4);
    col = 0;
  }
  __device__ __forceinline__ void next(uint2 (&a)[25]) {
#pragma unroll
    for (int q = 0; q < 21; q++) a[q] = col + 4 * q < N ? row[col / 4 + q] : make_uint2(0u, 0u);
    col += 84;
  }
};

// AES-128 (FIPS 197) tables, evaluated at compile time from the definitions: the S-box is
// the inverse in GF(2^8) mod x^8 + x^4 + x^3 + x + 1 followed by the affine map (constant
// 0x63); te[x] holds MixColumns' first column times S(x) as bytes (2S, S, S, 3S), so a
// round column is te[.] ^ rotl8(te[.]) ^ rotl16(te[.]) ^ rotl24(te[.]) ^ key, and S(x) is
// byte 1 of te[x].
namespace aes {
__host__ __device__ constexpr uint32_t xt(uint32_t a) { return ((a << 1) ^ ((a & 0x80u) ? 0x1Bu : 0u)) & 0xFFu; }
constexpr uint32_t gmul(uint32_t a, uint32_t b) {
  uint32_t r = 0;
  for (int i = 0; i < 8; i++) {
    if (b & 1u) r ^= a;
    a = xt(a);
    b >>= 1;
  }
  return r;
}
constexpr uint32_t ginv(uint32_t a) {  // a^254
  uint32_t r = 1, p = a;
  for (int e = 254; e; e >>= 1) {
    if (e & 1) r = gmul(r, p);
    p = gmul(p, p);
  }
  return a ? r : 0u;
}
constexpr uint32_t rotb(uint32_t b, int k) { return ((b << k) | (b >> (8 - k))) & 0xFFu; }
constexpr uint32_t sbox(uint32_t x) {
  const uint32_t b = ginv(x);
  return b ^ rotb(b, 1) ^ rotb(b, 2) ^ rotb(b, 3) ^ rotb(b, 4) ^ 0x63u;
}
struct Table {
  uint32_t te[256];
};
constexpr Table make_table() {
  Table t{};
  for (uint32_t x = 0; x < 256; x++) {
    const uint32_t s = sbox(x), s2 = xt(s);
    t.te[x] = s2 | (s << 8) | (s << 16) | ((s2 ^ s) << 24);
  }
  return t;
}
}  // namespace aes

static __constant__ aes::Table kAesTable = aes::make_table();

// C copies of the table, copy c of entry x at word x * C + c (bank c mod 32): with
// C = 32 every lane reads its own bank, with C = 16 lanes l and l + 16 may meet.
template <int C>
struct AesRows {
  static constexpr int SMEM = 256 * C * 4 + 52 * 4;
  const uint32_t *rk;  // 44 round-key words (LE columns), 4 round-1 constants, the entry stride
  uint32_t base;       // shared-window address of this lane's table copy
  uint32_t stride;     // 4 C, read back from shared memory so it stays a multiplier
  uint32_t row, cb, odd, r0, r3;
  uint2 carry;

  __device__ __forceinline__ static uint32_t rot8(uint32_t x) { return __funnelshift_l(x, x, 8); }
  __device__ __forceinline__ static uint32_t rot16(uint32_t x) { return __funnelshift_l(x, x, 16); }
  __device__ __forceinline__ static uint32_t rot24(uint32_t x) { return __funnelshift_l(x, x, 24); }
  // Table entry for byte K of w: one PRMT (the byte into the low position, zeros above)
  // and one IMAD (address = byte * stride + base) on the FMA pipe, which the Keccak-style
  // ALU-bound loop leaves idle.
  template <int K>
  __device__ __forceinline__ uint32_t tb(uint32_t w) const {
    const uint32_t b = prmt(w, 0u, 0x4440 | K);
    uint32_t a, v;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(a) : "r"(b), "r"(stride), "r"(base));
    asm volatile("ld.shared.u32 %0, [%1];" : "=r"(v) : "r"(a));
    return v;
  }
  __device__ __forceinline__ static uint32_t cte(uint32_t x) { return kAesTable.te[x]; }

  // Key schedule (one thread), then the round-1 terms that depend on the key alone: the
  // input block's words 1..3 are zero, so three of the four table terms of every round-1
  // column are constants of the instance.
  __device__ static void expand(const uint8_t *seed, uint32_t *k) {
    for (int i = 0; i < 4; i++)
      k[i] = seed[4 * i] | (seed[4 * i + 1] << 8) | (seed[4 * i + 2] << 16) | ((uint32_t)seed[4 * i + 3] << 24);
    uint32_t rc = 1;
    for (int i = 4; i < 44; i++) {
      uint32_t t = k[i - 1];
      if ((i & 3) == 0) {
        t = (t >> 8) | (t << 24);  // RotWord: bytes (a0 a1 a2 a3) -> (a1 a2 a3 a0)
        t = ((cte(t & 0xFFu) >> 8) & 0xFFu) | (cte((t >> 8) & 0xFFu) & 0xFF00u) |
            ((cte((t >> 16) & 0xFFu) << 8) & 0xFF0000u) | ((cte(t >> 24) << 16) & 0xFF000000u);  // SubWord
        t ^= rc;
        rc = aes::xt(rc);
      }
      k[i] = k[i - 4] ^ t;
    }
    const uint32_t s1 = k[1], s2 = k[2], s3 = k[3];
    k[44] = rot8(cte((s1 >> 8) & 0xFFu)) ^ rot16(cte((s2 >> 16) & 0xFFu)) ^ rot24(cte(s3 >> 24)) ^ k[4];
    k[45] = cte(s1 & 0xFFu) ^ rot8(cte((s2 >> 8) & 0xFFu)) ^ rot16(cte((s3 >> 16) & 0xFFu)) ^ k[5];
    k[46] = cte(s2 & 0xFFu) ^ rot8(cte((s3 >> 8) & 0xFFu)) ^ rot24(cte(s1 >> 24)) ^ k[6];
    k[47] = cte(s3 & 0xFFu) ^ rot16(cte((s1 >> 16) & 0xFFu)) ^ rot24(cte(s2 >> 24)) ^ k[7];
  }

  __device__ __forceinline__ void setup(const uint8_t *seed, uint8_t *mem) {
    uint32_t *tab = reinterpret_cast<uint32_t *>(mem);
    uint32_t *k = tab + 256 * C;
    for (int i = threadIdx.x; i < 256 * C; i += blockDim.x) tab[i] = kAesTable.te[i / C];
    if (threadIdx.x == 0) {
      expand(seed, k);
      k[48] = 4 * C;
    }
    base = smem_u32(tab + (threadIdx.x & 31) % C);
    rk = k;
  }

  __device__ __forceinline__ void start(uint2 (&)[25], uint32_t j) {
    row = j;
    cb = 0;
    odd = 0;
    stride = *reinterpret_cast<const volatile uint32_t *>(rk + 48);
    const uint32_t s0 = j ^ rk[0];  // bytes 0 and 1 of the first state word depend on the row only
    r0 = rk[44] ^ tb<0>(s0);
    r3 = rk[47] ^ rot8(tb<1>(s0));
  }

  // Bytes S(b0(a)), S(b1(b)), S(b2(c)), S(b3(d)) of the last round.
  __device__ __forceinline__ uint32_t last(uint32_t a, uint32_t b, uint32_t c, uint32_t d) const {
    const uint32_t lo = prmt(tb<0>(a), tb<1>(b), 0x0051);
    const uint32_t hi = prmt(tb<2>(c), tb<3>(d), 0x5100);
    return prmt(lo, hi, 0x7610);
  }

  // AES-128 of LE16(row) || LE16(8 c) || 0^12.
  __device__ __forceinline__ uint4 block(uint32_t c) const {
    const uint32_t s0 = (row | ((8u * c) << 16)) ^ rk[0];
    uint32_t t0 = r0, t1 = rk[45] ^ rot24(tb<3>(s0)), t2 = rk[46] ^ rot16(tb<2>(s0)), t3 = r3;
#pragma unroll
    for (int r = 2; r < 10; r++) {
      const uint4 k = *reinterpret_cast<const uint4 *>(rk + 4 * r);
      const uint32_t u0 = tb<0>(t0) ^ rot8(tb<1>(t1)) ^ rot16(tb<2>(t2)) ^ rot24(tb<3>(t3)) ^ k.x;
      const uint32_t u1 = tb<0>(t1) ^ rot8(tb<1>(t2)) ^ rot16(tb<2>(t3)) ^ rot24(tb<3>(t0)) ^ k.y;
      const uint32_t u2 = tb<0>(t2) ^ rot8(tb<1>(t3)) ^ rot16(tb<2>(t0)) ^ rot24(tb<3>(t1)) ^ k.z;
      const uint32_t u3 = tb<0>(t3) ^ rot8(tb<1>(t0)) ^ rot16(tb<2>(t1)) ^ rot24(tb<3>(t2)) ^ k.w;
      t0 = u0;
      t1 = u1;
      t2 = u2;
      t3 = u3;
    }
    const uint4 k = *reinterpret_cast<const uint4 *>(rk + 40);
    return make_uint4(last(t0, t1, t2, t3) ^ k.x, last(t1, t2, t3, t0) ^ k.y, last(t2, t3, t0, t1) ^ k.z,
                      last(t3, t0, t1, t2) ^ k.w);
  }

  __device__ __forceinline__ void next(uint2 (&a)[25]) {
    uint2 buf[22];
    const uint32_t nb = odd ? 10u : 11u;
#pragma unroll 1
    for (uint32_t b = 0; b < nb; b++) {
      const uint4 c = block(cb + b);
      buf[2 * b] = make_uint2(c.x, c.y);
      buf[2 * b + 1] = make_uint2(c.z, c.w);
    }
    cb += nb;
    if (odd) {
      a[0] = carry;
#pragma unroll
      for (int q = 0; q < 20; q++) a[q + 1] = buf[q];
    } else {
#pragma unroll
      for (int q = 0; q < 21; q++) a[q] = buf[q];
      carry = buf[21];
    }
    odd ^= 1u;
  }
};
using AesRowsFull = AesRows<32>;  // every lane its own bank
using AesRowsHalf = AesRows<16>;  // half the shared memory (the dp4a / INT32 S'A stage)

// V = S'B + E'' + Encode(mu): 64 outputs over 976 terms, 256 threads.  sval(k, j) yields
// S'[k][j] sign-extended; C is written to ct (encaps) or compared with it (decaps).
template <int MODE, typename SVal>
__device__ __forceinline__ uint32_t finish_c(const Inst &v, SVal sval, uint32_t (*red)[64]) {
  const int tid = threadIdx.x, o = tid & 63, q = tid >> 6, k = o >> 3, l = o & 7;
  const uint8_t *bsrc = MODE == OP_ENC ? v.pk + SEEDA : v.sk + LENS + SEEDA;
  uint32_t acc = 0;
  for (int j = 244 * q; j < 244 * q + 244; j++) {
    const uint32_t bv = ((uint32_t)bsrc[2 * (NBAR * j + l)] << 8) | bsrc[2 * (NBAR * j + l) + 1];
    acc += (uint32_t)sval(k, j) * bv;
  }
  red[q][o] = acc;
  __syncthreads();
  uint32_t diff = 0;
  if (tid < 64) {
    const uint16_t *epp = v.rw + 2 * N * NBAR;
    const uint8_t *mu = MODE == OP_ENC ? v.coins : v.mu;
    const int kr = tid >> 3, lc = tid & 7;
    const uint32_t t3 = mu[3 * kr] | ((uint32_t)mu[3 * kr + 1] << 8) | ((uint32_t)mu[3 * kr + 2] << 16);
    const uint32_t enc = ((t3 >> (3 * lc)) & 7u) << 13;
    const uint32_t c = (red[0][tid] + red[1][tid] + red[2][tid] + red[3][tid] + epp[tid] + enc) & 0xFFFFu;
    uint8_t *dst = v.ct + PKB + 2 * tid;
    if (MODE == OP_ENC) {
      dst[0] = (uint8_t)(c >> 8);
      dst[1] = (uint8_t)c;
    } else {
      diff = c ^ (((uint32_t)dst[0] << 8) | dst[1]);
    }
  }
  return diff;
}

// ---------------------------------------------------------------- B' = S'A + E', dp2a form
// Each warp owns 32-row chunks of A (lane = row).  After every squeeze the warp's
// 32 x 84 tile goes to shared memory and the warp forms row-pair x S' dot products with
// dp2a (16-bit A halves x 8-bit S'), flushing column partial sums with shared atomics.
constexpr int DP4A_SMEM = 83200 + 4 * 64 * 4;

// I32 = true is the plain INT32 form (FrodoKEM976-GPU/src/matrix_kernel.cu:75-111, the
// reference's non-DP path): the same tiles, 32-bit multiply-adds instead of dp2a.
template <int MODE, bool I32 = false, class G = ShakeRows>
__device__ __forceinline__ void sa_dp4a_cta(const Inst &v, uint8_t *smem) {
  uint32_t *acc = reinterpret_cast<uint32_t *>(smem);             // [8][976]
  uint32_t *sp8 = reinterpret_cast<uint32_t *>(smem + 31232);     // [248 quads][8 k]: S'[k][4q..4q+3]
  uint32_t *tile = reinterpret_cast<uint32_t *>(smem + 39168);    // [8 warps][32 rows][43]
  uint32_t(*red)[64] = reinterpret_cast<uint32_t(*)[64]>(smem + 83200);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint16_t *rw = v.rw;
  const uint8_t *seed = v.amat ? reinterpret_cast<const uint8_t *>(v.amat) : MODE == OP_ENC ? v.pk : v.sk + LENS;
  for (int q = tid; q < N * NBAR; q += 256) acc[q] = 0;
  for (int q = tid; q < (ROWS_PAD / 4) * NBAR; q += 256) {
    const int qd = q >> 3, k = q & 7;
    uint32_t s = 0;
    if (4 * qd < N) {
      const uint2 x = *reinterpret_cast<const uint2 *>(rw + k * N + 4 * qd);
      s = prmt(x.x, x.y, 0x6420);
    }
    sp8[q] = s;
  }
  G gen;
  gen.setup(seed, smem + DP4A_SMEM);
  __syncthreads();
  uint32_t *mt = tile + warp * 32 * 43;
  for (int c = warp; c < ROWS_PAD / 32; c += 8) {
    uint2 a[25];
    gen.start(a, 32 * c + lane);
    for (int blk = 0; blk < 12; blk++) {
      gen.next(a);
#pragma unroll
      for (int q = 0; q < 21; q++) {
        mt[lane * 43 + 2 * q] = a[q].x;
        mt[lane * 43 + 2 * q + 1] = a[q].y;
      }
      __syncwarp();
      const int ncw = blk < 11 ? 42 : 26;
      for (int w = lane; w < ncw; w += 32) {
        int alo[8], ahi[8];
#pragma unroll
        for (int k = 0; k < 8; k++) alo[k] = ahi[k] = 0;
#pragma unroll 2
        for (int rq = 0; rq < 8; rq++) {
          const uint32_t x0 = mt[(4 * rq) * 43 + w], x1 = mt[(4 * rq + 1) * 43 + w];
          const uint32_t x2 = mt[(4 * rq + 2) * 43 + w], x3 = mt[(4 * rq + 3) * 43 + w];
          const int p01l = prmt(x0, x1, 0x5410), p01h = prmt(x0, x1, 0x7632);
          const int p23l = prmt(x2, x3, 0x5410), p23h = prmt(x2, x3, 0x7632);
          const uint4 s0 = *reinterpret_cast<const uint4 *>(sp8 + (8 * c + rq) * 8);
          const uint4 s1 = *reinterpret_cast<const uint4 *>(sp8 + (8 * c + rq) * 8 + 4);
          const int sv[8] = {(int)s0.x, (int)s0.y, (int)s0.z, (int)s0.w, (int)s1.x, (int)s1.y, (int)s1.z, (int)s1.w};
          if (I32) {
            const uint32_t xr[4] = {x0, x1, x2, x3};
#pragma unroll
            for (int r = 0; r < 4; r++) {
              const int lo = (int)(xr[r] & 0xFFFFu), hi = (int)(xr[r] >> 16);
#pragma unroll
              for (int k = 0; k < 8; k++) {
                const int sk = (int)(int8_t)(sv[k] >> (8 * r));
                alo[k] += lo * sk;
                ahi[k] += hi * sk;
              }
            }
          } else {
#pragma unroll
            for (int k = 0; k < 8; k++) {
              alo[k] = dp2a_hi(p23l, sv[k], dp2a_lo(p01l, sv[k], alo[k]));
              ahi[k] = dp2a_hi(p23h, sv[k], dp2a_lo(p01h, sv[k], ahi[k]));
            }
          }
        }
        const int i0 = 84 * blk + 2 * w;
#pragma unroll
        for (int k = 0; k < 8; k++) {
          atomicAdd(&acc[k * N + i0], (uint32_t)alo[k]);
          atomicAdd(&acc[k * N + i0 + 1], (uint32_t)ahi[k]);
        }
      }
      __syncwarp();
    }
  }
  __syncthreads();
  uint32_t diff = 0;
  for (int p = tid; p < N * NBAR / 2; p += 256) {
    const uint32_t v0 = acc[2 * p] + rw[N * NBAR + 2 * p], v1 = acc[2 * p + 1] + rw[N * NBAR + 2 * p + 1];
    const uint32_t packed = bswap16x2(v0, v1);
    if (MODE == OP_ENC) *reinterpret_cast<uint32_t *>(v.ct + 4 * p) = packed;
    else diff |= packed ^ *reinterpret_cast<const uint32_t *>(v.ct + 4 * p);
  }
  auto sval = [&](int k, int j) -> int32_t {
    return (int32_t)(int8_t)(uint8_t)(sp8[(j >> 2) * 8 + k] >> (8 * (j & 3)));
  };
  diff |= finish_c<MODE>(v, sval, red);
  const int any = __syncthreads_or(diff != 0);
  if (MODE == OP_DEC && tid == 0) *v.fail = (uint32_t)any;
}

// ---------------------------------------------------------------- B' = S'A + E', tcgen05 form
// A (976 x 976, u16) is consumed as u8 hi/lo limb planes.  GEMM view per squeeze block
// blk (columns 84*blk .. +83 of A):  D_blk,limb[m][k] += sum_j limb(A[j][84 blk + m]) S'[k][j],
// M = 128 (84 valid), N = 8, K = 32 rows per MMA.  The limb tile is MN-major (row j of
// A is contiguous along M) in the canonical no-swizzle layout: byte (m, j) at
// (m/16)*512 + (j/8)*128 + (j%8)*16 + m%16.  S'^T is the K-major B operand: byte (j, k) at
// (j/16)*128 + k*16 + j%16.  24 accumulators (12 blocks x 2 limbs) x 8 columns in TMEM;
// B' = lo + 256 hi (mod 2^16).  Every producer warp issues its own MMAs and commits
// them to its stage barrier; the tile ring has NST stages per warp.
constexpr int TC_SP_BYTES = 62 * 128;
// A tile stage: a warp's 32 squeezed blocks as an MN-major u8 operand, M = the block's 168
// bytes in stream order (11 M-chunks of 16 bytes x 32 rows, 512 bytes each).
constexpr int TC_STAGE = 6144;
constexpr int TC_TMEM_COLS = 256;

template <int NST>
struct TcLayout {
  static constexpr int ring = TC_SP_BYTES;
  // +2 KB: the second MMA of a stage reads M-chunks 8..15, up to 8 KB past the stage start
  static constexpr int bars = ring + 8 * NST * TC_STAGE + 2048;
  static constexpr int tslot = bars + (8 * NST + 1) * 8;
  static constexpr int red = (tslot + 4 + 15) & ~15;
  static constexpr int total = red + 4 * 64 * 4;
};

// TMEM columns [tbase, tbase + 192) must be allocated by the caller.  Returns false if a
// bounded wait expired (the error word is set; the CTA still leaves TMEM idle).
template <int MODE, int NST, class G = ShakeRows>
__device__ __forceinline__ bool sa_tc_cta(const Inst &v, uint8_t *smem, uint32_t tbase, uint32_t *err) {
  using L = TcLayout<NST>;
  uint8_t *sp = smem;
  uint8_t *ring = smem + L::ring;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + L::bars);
  uint32_t(*red)[64] = reinterpret_cast<uint32_t(*)[64]>(smem + L::red);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint16_t *rw = v.rw;
  const uint8_t *seed = v.amat ? reinterpret_cast<const uint8_t *>(v.amat) : MODE == OP_ENC ? v.pk : v.sk + LENS;

  for (int q = tid; q < 62 * NBAR; q += 256) {
    const int g = q >> 3, k = q & 7;
    uint4 o = make_uint4(0, 0, 0, 0);
    if (16 * g < N) {
      const uint4 x0 = *reinterpret_cast<const uint4 *>(rw + k * N + 16 * g);
      const uint4 x1 = *reinterpret_cast<const uint4 *>(rw + k * N + 16 * g + 8);
      o = make_uint4(prmt(x0.x, x0.y, 0x6420), prmt(x0.z, x0.w, 0x6420), prmt(x1.x, x1.y, 0x6420),
                     prmt(x1.z, x1.w, 0x6420));
    }
    *reinterpret_cast<uint4 *>(sp + g * 128 + k * 16) = o;
  }
  if (tid == 0) {
    for (int q = 0; q < 8 * NST; q++) mbar_init(&bars[q], 1);
    mbar_init(&bars[8 * NST], 8);
    fence_mbar_init();
  }
  G gen;
  gen.setup(seed, smem + L::total);
  if (warp < 4) {
#pragma unroll
    for (int col = 0; col < 192; col += 16) tmem_st16_zero(tbase + ((uint32_t)(warp * 32) << 16) + col);
    tmem_wait_st();
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();

  constexpr uint32_t idesc = idesc_i8(128, 8, false, true, true, false);
  const uint32_t sp_addr = smem_u32(sp);
  const int roff = (lane >> 3) * 128 + (lane & 7) * 16;
  bool ok = true;
  uint32_t u = 0;
  for (int c = warp; c < ROWS_PAD / 32; c += 8) {
    uint2 a[25];
    gen.start(a, 32 * c + lane);
    const uint64_t bdesc = sdesc(sp_addr + 256 * c, 128, 1024);
    for (int blk = 0; blk < 12; blk++, u++) {
      gen.next(a);
      const int s = u % NST;
      if (u >= NST && ok) ok = mbar_wait(&bars[warp * NST + s], ((u / NST) - 1) & 1);
      ok = __all_sync(0xffffffffu, ok);
      uint8_t *stg = ring + (warp * NST + s) * TC_STAGE;
      // The block's bytes as squeezed: entry e is M-row 2e (low byte) and 2e + 1 (high byte),
      // so the u8 limbs need no byte permutes; the epilogue pairs the two rows' sums.
#pragma unroll
      for (int cc = 0; cc < 10; cc++)
        *reinterpret_cast<uint4 *>(stg + cc * 512 + roff) =
            make_uint4(a[2 * cc].x, a[2 * cc].y, a[2 * cc + 1].x, a[2 * cc + 1].y);
      *reinterpret_cast<uint2 *>(stg + 10 * 512 + roff) = a[20];
      fence_proxy_async_smem();
      __syncwarp();
      if (lane == 0 && ok) {
        tc_fence_after();
        const uint32_t sa = smem_u32(stg);
        mma_i8(tbase + blk * 16, sdesc(sa, 128, 512), bdesc, idesc, 1u);             // entries 0..63
        mma_i8(tbase + blk * 16 + 8, sdesc(sa + 4096, 128, 512), bdesc, idesc, 1u);  // entries 64..83
        mma_commit(&bars[warp * NST + s]);
      }
      __syncwarp();
    }
  }
  if (lane == 0) mma_commit(&bars[8 * NST]);
  // 31 row groups over 8 warps: warp 7 runs out of rows a group early.  It waits in the
  // hardware barrier, which issues nothing, not in an mbarrier poll loop whose compares and
  // branches would take ALU slots from the warps still hashing.
  __syncthreads();
  bool fin = mbar_wait(&bars[8 * NST], 0);
  // Drain: observe each stage barrier's last phase, so no arrival is still pending
  // when the barriers are initialised again for the next instance.
  for (int s = 0; s < NST; s++)
    if (ok && u > (uint32_t)s) fin &= mbar_wait(&bars[warp * NST + s], ((u - 1 - s) / NST) & 1);
  if ((!fin || !ok) && lane == 0) atomicOr(err, DEV_ERR_TIMEOUT);
  tc_fence_after();

  // Epilogue: B'[k][84 blk + e] = lo + 256 hi + E' (mod 2^16).  TMEM lane 2e holds the
  // low-byte sums of entry e, lane 2e + 1 the high-byte sums: columns 0..7 entries 0..63,
  // columns 8..15 entries 64..83 (lanes 0..39).  Even lanes take the pair's result.
  uint32_t diff = 0;
  const int qd = warp & 3, t = qd * 32 + lane, b0 = warp < 4 ? 0 : 6;
  for (int blk = b0; blk < b0 + 6; blk++) {
    uint32_t r[16];
    tmem_ld16(tbase + ((uint32_t)(qd * 32) << 16) + blk * 16, r);
    tmem_wait_ld();
#pragma unroll
    for (int q = 0; q < 16; q++) r[q] += __shfl_down_sync(0xffffffffu, r[q], 1) << 8;
    const int valid = blk < 11 ? 84 : 52;
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int e = 64 * h + (t >> 1);
      if ((lane & 1) == 0 && e < valid && (h == 0 || t < 40)) {
        const int col = 84 * blk + e;
#pragma unroll
        for (int k = 0; k < 8; k++) {
          const uint32_t x = (r[8 * h + k] + rw[N * NBAR + k * N + col]) & 0xFFFFu;
          uint8_t *d = v.ct + 2 * (k * N + col);
          if (MODE == OP_ENC) {
            *reinterpret_cast<uint16_t *>(d) = (uint16_t)((x >> 8) | (x << 8));
          } else {
            diff |= x ^ (((uint32_t)d[0] << 8) | d[1]);
          }
        }
      }
    }
  }
  auto sval = [&](int k, int j) -> int32_t {
    return (int32_t)(int8_t)sp[(j >> 4) * 128 + k * 16 + (j & 15)];
  };
  tc_fence_before();
  __syncthreads();
  if (tid == 0 && ok && fin)  // all arrivals observed: the barrier memory may be reused by the next task
    for (int q = 0; q < 8 * NST + 1; q++) mbar_inval(&bars[q]);
  diff |= finish_c<MODE>(v, sval, red);
  const int any = __syncthreads_or(diff != 0);
  if (MODE == OP_DEC && tid == 0) *v.fail = (uint32_t)any;
  return ok && fin;
}

// ---------------------------------------------------------------- B = A S + E (keypair), dp2a form
// Thread = row of A: after each squeeze the thread dots its 84 fresh columns with the
// 8 rows of S^T (broadcast from shared memory), so B[j][k] accumulates in registers.
constexpr int KP_AS_SMEM = 12 * 21 * 8 * 4;

template <bool I32 = false, class G = ShakeRows>
__device__ __forceinline__ void kp_as_dp4a_cta(const Inst &v, uint8_t *smem) {
  uint32_t *st8 = reinterpret_cast<uint32_t *>(smem);  // [blk][q][k]: S^T[k][84 blk + 4q .. +3]
  const int tid = threadIdx.x;
  const uint16_t *rw = v.rw;
  for (int x = tid; x < 12 * 21 * 8; x += 256) {
    const int k = x & 7, q = (x >> 3) % 21, blk = x / 168, j = 84 * blk + 4 * q;
    uint32_t s = 0;
    if (j < N) {
      const uint2 y = *reinterpret_cast<const uint2 *>(rw + k * N + j);
      s = prmt(y.x, y.y, 0x6420);
    }
    st8[x] = s;
  }
  G gen;
  gen.setup(v.pk, smem + KP_AS_SMEM);
  __syncthreads();
  for (int j = tid; j < N; j += 256) {
    uint2 a[25];
    gen.start(a, j);
    int acc[8];
#pragma unroll
    for (int k = 0; k < 8; k++) acc[k] = 0;
    for (int blk = 0; blk < 12; blk++) {
      gen.next(a);
#pragma unroll
      for (int q = 0; q < 21; q++) {
        const uint4 s0 = *reinterpret_cast<const uint4 *>(st8 + (blk * 21 + q) * 8);
        const uint4 s1 = *reinterpret_cast<const uint4 *>(st8 + (blk * 21 + q) * 8 + 4);
        const int sv[8] = {(int)s0.x, (int)s0.y, (int)s0.z, (int)s0.w, (int)s1.x, (int)s1.y, (int)s1.z, (int)s1.w};
        if (I32) {
          const int c0 = (int)(a[q].x & 0xFFFFu), c1 = (int)(a[q].x >> 16), c2 = (int)(a[q].y & 0xFFFFu),
                    c3 = (int)(a[q].y >> 16);
#pragma unroll
          for (int k = 0; k < 8; k++)
            acc[k] += c0 * (int)(int8_t)sv[k] + c1 * (int)(int8_t)(sv[k] >> 8) + c2 * (int)(int8_t)(sv[k] >> 16) +
                      c3 * (sv[k] >> 24);
        } else {
#pragma unroll
          for (int k = 0; k < 8; k++) acc[k] = dp2a_hi((int)a[q].y, sv[k], dp2a_lo((int)a[q].x, sv[k], acc[k]));
        }
      }
    }
    uint32_t x[8];
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = (uint32_t)acc[k] + rw[N * NBAR + NBAR * j + k];
    const uint4 o = make_uint4(bswap16x2(x[0], x[1]), bswap16x2(x[2], x[3]), bswap16x2(x[4], x[5]),
                               bswap16x2(x[6], x[7]));
    *reinterpret_cast<uint4 *>(v.pk + SEEDA + 16 * j) = o;
    *reinterpret_cast<uint2 *>(v.sk + LENS + SEEDA + 16 * j) = make_uint2(o.x, o.y);
    *reinterpret_cast<uint2 *>(v.sk + LENS + SEEDA + 16 * j + 8) = make_uint2(o.z, o.w);
  }
  __syncthreads();
}


// ---------------------------------------------------------------- B = A S + E (keypair), tcgen05 form
// GEMM view: D[i][k] = sum_j limb(A[i][j]) S^T[k][j], M = 128 rows of A per tile (a
// warpgroup, thread = row), N = 8, K = the 84 columns of one squeeze block padded to 96
// (3 K steps; S^T is zero-padded so the pad bytes contribute nothing).  A limb tiles are
// K-major (row i contiguous along K, as the sponge squeezes it): byte (i, kk) at
// (i/8)*768 + (kk/16)*128 + (i%8)*16 + kk%16.  S^T per block is the K-major B operand:
// byte (kk, k) at (kk/16)*128 + k*16 + kk%16.  The two warpgroups take M tiles g, g+2, g+4,
// g+6 (tile 7 holds rows 896..1023; rows >= 976 are computed and discarded); each has its
// own 2-stage ring, TMEM columns [32g, 32g+16) and named barrier 1+g.
constexpr int KPT_ST_BLK = 6 * 128;                // S^T operand per block (96 K bytes x 8 rows)
constexpr int KPT_PLANE = 16 * 768;                // one limb plane of a 128-row tile
constexpr int KPT_STAGE = 2 * KPT_PLANE;
constexpr int KPT_NST = 2;
template <int NST>
struct KptLayoutT {
  static constexpr int st = 0;
  static constexpr int ring = 12 * KPT_ST_BLK;                   // 9216
  static constexpr int bars = ring + 2 * NST * KPT_STAGE;        // per warpgroup: NST stage + 1 tile
  static constexpr int total = bars + 2 * (NST + 1) * 8;
};
using KptLayout = KptLayoutT<KPT_NST>;

__device__ __forceinline__ void wg_sync(int g) {
  asm volatile("bar.sync %0, 128;" ::"r"(1 + g) : "memory");
}

// TMEM columns [tbase, tbase + 48) must be allocated by the caller.
template <int NST = KPT_NST, class G = ShakeRows>
__device__ __forceinline__ bool kp_as_tc_cta(const Inst &v, uint8_t *smem, uint32_t tbase, uint32_t *err) {
  using L = KptLayoutT<NST>;
  const int tid = threadIdx.x, warp = tid >> 5, g = warp >> 2, l = tid & 127;
  uint8_t *stop = smem + L::st;
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + L::bars) + g * (NST + 1);
  const uint16_t *rw = v.rw;
  // S^T operand of every block, zero-padded to 96 columns.
  for (int x = tid; x < 12 * 8 * 6; x += 256) {
    const int blk = x / 48, k = (x / 6) % 8, q = x % 6;
    uint32_t w[4] = {0, 0, 0, 0};
#pragma unroll
    for (int c = 0; c < 16; c++) {
      const int kk = 16 * q + c, j = 84 * blk + kk;
      const uint32_t sv = (kk < 84 && j < N) ? (uint32_t)(rw[k * N + j] & 0xFFu) : 0u;
      w[c >> 2] |= sv << (8 * (c & 3));
    }
    *reinterpret_cast<uint4 *>(stop + blk * KPT_ST_BLK + q * 128 + k * 16) = make_uint4(w[0], w[1], w[2], w[3]);
  }
  if (l == 0) {
    for (int q = 0; q < NST + 1; q++) mbar_init(&bars[q], 1);
    fence_mbar_init();
  }
  G gen;
  gen.setup(v.pk, smem + L::total);
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();

  constexpr uint32_t idesc = idesc_i8(128, 8, false, true, false, false);
  const uint32_t st_addr = smem_u32(stop);
  uint8_t *ring = smem + L::ring + g * NST * KPT_STAGE;
  const uint32_t tcol = tbase + 32 * g;
  const int roff = (l >> 3) * 768 + (l & 7) * 16;
  bool ok = true;
  uint32_t u = 0, tiles = 0;
  for (int t = g; t < 8; t += 2, tiles++) {
    const int i = 128 * t + l;
    uint2 a[25];
    gen.start(a, i);
    for (int blk = 0; blk < 12; blk++, u++) {
      gen.next(a);
      uint32_t lo[21], hi[21];
#pragma unroll
      for (int q = 0; q < 21; q++) {
        lo[q] = prmt(a[q].x, a[q].y, 0x6420);
        hi[q] = prmt(a[q].x, a[q].y, 0x7531);
      }
      const int s = u % NST;
      if (u >= NST && ok) ok = mbar_wait(&bars[s], ((u / NST) - 1) & 1);
      uint8_t *stg = ring + s * KPT_STAGE;
#pragma unroll
      for (int q = 0; q < 5; q++) {
        *reinterpret_cast<uint4 *>(stg + roff + q * 128) = make_uint4(lo[4 * q], lo[4 * q + 1], lo[4 * q + 2], lo[4 * q + 3]);
        *reinterpret_cast<uint4 *>(stg + KPT_PLANE + roff + q * 128) =
            make_uint4(hi[4 * q], hi[4 * q + 1], hi[4 * q + 2], hi[4 * q + 3]);
      }
      *reinterpret_cast<uint4 *>(stg + roff + 5 * 128) = make_uint4(lo[20], 0u, 0u, 0u);
      *reinterpret_cast<uint4 *>(stg + KPT_PLANE + roff + 5 * 128) = make_uint4(hi[20], 0u, 0u, 0u);
      fence_proxy_async_smem();
      wg_sync(g);
      if (l == 0 && ok) {
        tc_fence_after();
        const uint32_t sa = smem_u32(stg);
#pragma unroll
        for (int ks = 0; ks < 3; ks++) {
          const uint64_t bd = sdesc(st_addr + blk * KPT_ST_BLK + ks * 256, 128, 1024);
          const uint32_t acc = (blk | ks) ? 1u : 0u;
          mma_i8(tcol, sdesc(sa + ks * 256, 128, 768), bd, idesc, acc);
          mma_i8(tcol + 8, sdesc(sa + KPT_PLANE + ks * 256, 128, 768), bd, idesc, acc);
        }
        mma_commit(&bars[s]);
      }
    }
    if (l == 0) mma_commit(&bars[NST]);
    const bool fin = mbar_wait(&bars[NST], tiles & 1);
    if (!fin) ok = false;
    tc_fence_after();
    uint32_t r[16];
    tmem_ld16(tcol + ((uint32_t)((warp & 3) * 32) << 16), r);
    tmem_wait_ld();
    if (i < N) {
      uint32_t x[8];
#pragma unroll
      for (int k = 0; k < 8; k++) x[k] = r[k] + (r[8 + k] << 8) + rw[N * NBAR + NBAR * i + k];
      const uint2 o0 = make_uint2(bswap16x2(x[0], x[1]), bswap16x2(x[2], x[3]));
      const uint2 o1 = make_uint2(bswap16x2(x[4], x[5]), bswap16x2(x[6], x[7]));
      *reinterpret_cast<uint2 *>(v.pk + SEEDA + 16 * i) = o0;
      *reinterpret_cast<uint2 *>(v.pk + SEEDA + 16 * i + 8) = o1;
      *reinterpret_cast<uint2 *>(v.sk + LENS + SEEDA + 16 * i) = o0;
      *reinterpret_cast<uint2 *>(v.sk + LENS + SEEDA + 16 * i + 8) = o1;
    }
    tc_fence_before();
    wg_sync(g);  // TMEM read before the next tile overwrites the accumulators
    tc_fence_after();
  }
  // Drain: observe each stage barrier's last phase before the barriers are invalidated.
  bool fin = true;
  for (int s = 0; s < NST; s++)
    if (ok && u > (uint32_t)s) fin &= mbar_wait(&bars[s], ((u - 1 - s) / NST) & 1);
  if ((!ok || !fin) && l == 0) atomicOr(err, DEV_ERR_TIMEOUT);
  tc_fence_before();
  __syncthreads();
  if (l == 0 && ok && fin)
    for (int q = 0; q < NST + 1; q++) mbar_inval(&bars[q]);
  __syncthreads();
  return ok && fin;
}

}  // namespace fdev
}  // namespace dpkem
