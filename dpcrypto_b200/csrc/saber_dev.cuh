// Saber (LightSaber l=2, Saber l=3, FireSaber l=4) device routines for sm_100a, written per
// instance so the batched kernels (saber.cu) and the persistent mixed-batch kernel
// (mixed.cu) run the same code.
//
// Kernel chain per operation:
//   prologue  (64 threads = 32 instances: warp 0 runs the hash chain and GenSecret's
//              SHAKE128 (decaps: then SHA3-256 of the input ciphertext), warp 1 runs
//              GenMatrix's SHAKE128, in parallel; raw XOF bytes go to the scratch arena)
//   product   (CTA/instance: CBD sampling, 13/10-bit unpacking, the negacyclic
//              matrix-vector and inner products, rounding, packing / comparison)
//   finish    (thread/instance: SHA3-256(c) (encaps), final key, or H(pk) for keypair)
// Decaps runs the product kernel twice: first the inner product v = b'^T s with the
// secret from sk (-> m'), then the re-encryption in compare mode.
//
// Two product forms:
//   dp4a: thread = output coefficient; dp2a(16-bit public pair, 8-bit secret pair)
//         over a reversed, sign-extended secret window (no branch on the wrap).
//   tc:   tcgen05.mma kind::i8, D[coef][(out, limb)] = sum_K H_j[coef][K] * P[K][(out,limb)].
//         The public polynomials are written in reversed coefficient order along K,
//         which turns the negacyclic Toeplitz block of each secret into a Hankel block:
//         T'[i][k'] = s_ext[i + k' - 255].  Its core matrix (8 rows x 16 bytes) at
//         (mi, ki) depends only on t = mi + 2 ki, so the whole 256 x 256 block is 62
//         distinct 128-byte core matrices (SBO = 128, LBO = 256) instead of 64 KB.
//         Public coefficients are split into u8 limbs (lo 8 bits, hi bits) along N.
//
// Replaces the reference's per-stage launches (SABER-GPU/src/cuda_kernel.cu:19-299),
// its dp4a-shaped DoDP4Av7/_inner products over HBM rotation tables
// (SABER-GPU/src/poly.cu:26-206) and its FO helpers (pack.cu:215-255), following the
// round-3 specification order (cmov of z before the final hash).
#pragma once
#include "common.cuh"
#include "keccak.cuh"
#include "keccak_pair.cuh"
#include "msponge.cuh"
#include "tc.cuh"

namespace dpkem {
namespace sdev {

using saber::EP;
using saber::EQ;
constexpr int SN = saber::N;

enum PMode : int { PM_KEYPAIR = 0, PM_ENC = 1, PM_DEC_CMP = 2, PM_DEC_INNER = 3 };

template <int L>
struct SP {
  static constexpr saber::Params p = saber::params(L);
  static constexpr int MU = p.mu, ET = p.et;
  static constexpr int POLYVEC = p.polyvec, POLYVECCOMP = p.polyveccomp, PK = p.pk, SK = p.sk, CT = p.ct;
  static constexpr int ARAW = L * L * EQ * SN / 8;  // GenMatrix bytes
  static constexpr int SRAW = L * MU * SN / 8;      // GenSecret bytes
  static constexpr uint32_t H1 = 1u << (EQ - EP - 1);
  static constexpr uint32_t H2 = (1u << (EP - 2)) - (1u << (EP - ET - 1)) + (1u << (EQ - EP - 1));
};

// Scratch offsets within one instance's record (all multiples of 16).
template <int L>
struct Scr {
  static constexpr int ARAW = 0;
  static constexpr int SRAW = (SP<L>::ARAW + 15) & ~15;
  static constexpr int KR = SRAW + ((SP<L>::SRAW + 15) & ~15);
  static constexpr int MTXT = KR + 64;
  static constexpr int HC = MTXT + 32;  // decaps: SHA3-256(c), hashed by the prologue
  static constexpr int BYTES = HC + 32;
};

// Pointers of one instance, already offset into the caller's arrays and the scratch arena.
struct Inst {
  const uint8_t *coins;  // keypair 96 B, enc 32 B
  uint8_t *pk, *sk, *ct, *ss;
  uint8_t *scr;          // this instance's scratch record (Scr<L>::BYTES)
  uint32_t *fail;
};

template <int L>
__device__ __forceinline__ Inst inst_of(const SaberBatch &b, int i, int op) {
  using P = SP<L>;
  Inst v;
  v.coins = b.coins ? b.coins + (size_t)i * (op == OP_KEYPAIR ? 96 : 32) : nullptr;
  v.pk = b.pk ? b.pk + (size_t)i * P::PK : nullptr;
  v.sk = b.sk ? b.sk + (size_t)i * P::SK : nullptr;
  v.ct = b.ct ? b.ct + (size_t)i * P::CT : nullptr;
  v.ss = b.ss ? b.ss + (size_t)i * 32 : nullptr;
  v.scr = b.scr + (size_t)i * Scr<L>::BYTES;
  v.fail = b.fail + i;
  return v;
}

// SHAKE128 of a 32-byte seed held in 4 lanes, squeezing `len` bytes (len % 8 == 0) to dst.
__device__ __forceinline__ void shake128_seed32(const uint2 (&seed)[4], uint8_t *dst, int len) {
  uint2 a[25];
  keccak_zero(a);
#pragma unroll
  for (int q = 0; q < 4; q++) a[q] = seed[q];
  absorb_finish<168>(a, 32, 0x1Fu);
  for (int off = 0;; off += 168) {
#pragma unroll
    for (int q = 0; q < 21; q++)
      if (off + 8 * q < len) *reinterpret_cast<uint2 *>(dst + off + 8 * q) = a[q];
    if (off + 168 >= len) break;
    keccak_f1600(a);
  }
}

// SHA3-256 of a whole byte string (length multiple of 8, 8-byte aligned).
__device__ __forceinline__ void sha3_256_msg(const uint8_t *p, int len, uint2 (&out)[4]) {
  uint2 a[25];
  keccak_zero(a);
  const int pos = absorb_aligned<136>(a, 0, p, len);
  absorb_finish<136>(a, pos, 0x06u);
#pragma unroll
  for (int q = 0; q < 4; q++) out[q] = a[q];
}

// SHA3-256 / SHA3-512 of 64 bytes held in lanes.
__device__ __forceinline__ void sha3_256_64(const uint2 (&m)[8], uint2 (&out)[4]) {
  uint2 a[25];
  keccak_zero(a);
#pragma unroll
  for (int q = 0; q < 8; q++) a[q] = m[q];
  absorb_finish<136>(a, 64, 0x06u);
#pragma unroll
  for (int q = 0; q < 4; q++) out[q] = a[q];
}
__device__ __forceinline__ void sha3_512_64(const uint2 (&m)[8], uint2 (&out)[8]) {
  uint2 a[25];
  keccak_zero(a);
#pragma unroll
  for (int q = 0; q < 8; q++) a[q] = m[q];
  absorb_finish<72>(a, 64, 0x06u);
#pragma unroll
  for (int q = 0; q < 8; q++) out[q] = a[q];
}

// ---------------------------------------------------------------- prologue
// role 0 = hash chain + GenSecret XOF, role 1 = GenMatrix XOF: the two independent sponges
// of one instance (the batched kernel runs them on different warps).
template <int L, int OP>
__device__ __forceinline__ void prologue_inst(const Inst &v, int role) {
  using P = SP<L>;
  using S = Scr<L>;
  uint8_t *scr = v.scr;
  if (role == 1) {
    uint2 seed[4];
    if (OP == OP_KEYPAIR) {
      // seed_A = SHAKE128(coins[0:32], 32), published in pk.
      uint2 a[25];
      keccak_zero(a);
#pragma unroll
      for (int q = 0; q < 4; q++) a[q] = ld_lane(v.coins + 8 * q);
      absorb_finish<168>(a, 32, 0x1Fu);
      uint8_t *pk = v.pk + P::POLYVECCOMP;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        seed[q] = a[q];
        *reinterpret_cast<uint2 *>(pk + 8 * q) = a[q];
      }
    } else {
      const uint8_t *src = OP == OP_ENC ? v.pk + P::POLYVECCOMP : v.sk + P::POLYVEC + P::POLYVECCOMP;
#pragma unroll
      for (int q = 0; q < 4; q++) seed[q] = ld_lane(src + 8 * q);
    }
    shake128_seed32(seed, scr + S::ARAW, P::ARAW);
    return;
  }
  uint2 seed[4];
  if (OP == OP_KEYPAIR) {
#pragma unroll
    for (int q = 0; q < 4; q++) seed[q] = ld_lane(v.coins + 32 + 8 * q);
  } else {
    uint2 buf[8], kr[8];
    if (OP == OP_ENC) {
      // m = SHA3-256(coins), H(pk), kr = SHA3-512(m || H(pk))  (cuda_kernel.cu:68-70)
      uint2 c8[8], h[4];
#pragma unroll
      for (int q = 0; q < 4; q++) c8[q] = ld_lane(v.coins + 8 * q);
#pragma unroll
      for (int q = 4; q < 8; q++) c8[q] = make_uint2(0, 0);
      uint2 a[25];
      keccak_zero(a);
#pragma unroll
      for (int q = 0; q < 4; q++) a[q] = c8[q];
      absorb_finish<136>(a, 32, 0x06u);
#pragma unroll
      for (int q = 0; q < 4; q++) buf[q] = a[q];
      sha3_256_msg(v.pk, P::PK, h);
#pragma unroll
      for (int q = 0; q < 4; q++) buf[4 + q] = h[q];
    } else {
      // m' from the inner-product pass, H(pk) stored in sk (cuda_kernel.cu:231-232)
      const uint8_t *hpk = v.sk + P::SK - 64;
#pragma unroll
      for (int q = 0; q < 4; q++) {
        buf[q] = ld_lane(scr + S::MTXT + 8 * q);
        buf[4 + q] = ld_lane(hpk + 8 * q);
      }
    }
    sha3_512_64(buf, kr);
    uint8_t *krp = scr + S::KR;
#pragma unroll
    for (int q = 0; q < 8; q++) *reinterpret_cast<uint2 *>(krp + 8 * q) = kr[q];
    if (OP == OP_ENC) {
#pragma unroll
      for (int q = 0; q < 4; q++) *reinterpret_cast<uint2 *>(scr + S::MTXT + 8 * q) = buf[q];
    }
#pragma unroll
    for (int q = 0; q < 4; q++) seed[q] = kr[4 + q];
  }
  shake128_seed32(seed, scr + S::SRAW, P::SRAW);
  if (OP == OP_DEC) {
    // H(c) of the input ciphertext does not wait for the products: hashing it here keeps
    // this role (15 permutations at l = 3) shorter than GenMatrix's, and the finish stage
    // down to one permutation.
    uint2 hc[4];
    sha3_256_msg(v.ct, P::CT, hc);
#pragma unroll
    for (int q = 0; q < 4; q++) *reinterpret_cast<uint2 *>(scr + S::HC + 8 * q) = hc[q];
  }
}

// GenMatrix (prologue role 1) on a lane pair (p = lane parity): its 10 / 23 / 40 permutations are
// the longest chain of the prologue.  live = false keeps a padding pair of a partial warp in
// step (its reads are valid, its writes are skipped).
template <int L, int OP>
__device__ __forceinline__ void matrix_pair(const Inst &v, int p, bool live) {
  using P = SP<L>;
  using S = Scr<L>;
  uint32_t a[25];
  kpair::zero(a);
  if (OP == OP_KEYPAIR) {
    // seed_A = SHAKE128(coins[0:32], 32), published in pk.
#pragma unroll
    for (int q = 0; q < 4; q++) a[q] = kpair::to_slice(ld_lane(v.coins + 8 * q), p);
    kpair::absorb_finish<168>(a, 32, 0x1Fu, p);
    uint32_t seed[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      seed[q] = a[q];
      const uint32_t h = kpair::from_slice(a[q], p);
      if (live) *reinterpret_cast<uint32_t *>(v.pk + P::POLYVECCOMP + 8 * q + 4 * p) = h;
    }
    kpair::zero(a);
#pragma unroll
    for (int q = 0; q < 4; q++) a[q] = seed[q];
  } else {
    const uint8_t *src = OP == OP_ENC ? v.pk + P::POLYVECCOMP : v.sk + P::POLYVEC + P::POLYVECCOMP;
#pragma unroll
    for (int q = 0; q < 4; q++) a[q] = kpair::to_slice(ld_lane(src + 8 * q), p);
  }
  kpair::absorb_finish<168>(a, 32, 0x1Fu, p);
  kpair::squeeze<168>(a, v.scr + S::ARAW, P::ARAW, p, live);
}

// Encaps finish on a lane pair: k = SHA3-256(kr[0:32] || SHA3-256(c)), the same bytes as
// finish_inst<L, OP_ENC>; 10 dependent permutations at l = 3.
template <int L>
__device__ __forceinline__ void finish_enc_pair(const Inst &v, int p, bool live) {
  using P = SP<L>;
  using S = Scr<L>;
  uint32_t a[25], hc[4];
  kpair::zero(a);
  const int pos = kpair::absorb_aligned<136>(a, 0, v.ct, P::CT, p);
  kpair::absorb_finish<136>(a, pos, 0x06u, p);
#pragma unroll
  for (int q = 0; q < 4; q++) hc[q] = a[q];
  kpair::zero(a);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    a[q] = kpair::to_slice(ld_lane(v.scr + S::KR + 8 * q), p);
    a[4 + q] = hc[q];
  }
  kpair::absorb_finish<136>(a, 64, 0x06u, p);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    const uint32_t h = kpair::from_slice(a[q], p);
    if (live) *reinterpret_cast<uint32_t *>(v.ss + 8 * q + 4 * p) = h;
  }
}

// ---------------------------------------------------------------- several lanes per state
// The same prologue roles and encaps / keypair finish with each sponge spread over several
// lanes (msponge.cuh: S = msp::Multi<5>, five lanes per state, or msp::Multi<1>, a warp per
// state): the bytes written are those of prologue_inst / finish_inst.  live = false keeps a
// state without an instance in step (reads stay in bounds, writes are skipped).
template <class S, int L, int OP>
__device__ __forceinline__ void prologue_multi(const Inst &v, const S &s, int role, bool live) {
  using P = SP<L>;
  using Q = Scr<L>;
  uint8_t *scr = v.scr;
  uint2 a[S::NS];
  msp::zero<S>(a);
  if (role == 1) {  // GenMatrix
    if (OP == OP_KEYPAIR) {  // seed_A = SHAKE128(coins[0:32], 32), published in pk
      msp::absorb_aligned<S, 168>(a, s, 0, v.coins, 32, live);
      msp::absorb_finish<S, 168>(a, s, 32, 0x1Fu);
      msp::store<S>(a, s, v.pk + P::POLYVECCOMP, 4, live);
      msp::keep<S>(a, s, 4);
    } else {
      const uint8_t *src = OP == OP_ENC ? v.pk + P::POLYVECCOMP : v.sk + P::POLYVEC + P::POLYVECCOMP;
      msp::absorb_aligned<S, 168>(a, s, 0, src, 32, live);
    }
    msp::absorb_finish<S, 168>(a, s, 32, 0x1Fu);
    msp::squeeze<S, 168>(a, s, scr + Q::ARAW, P::ARAW, live);
    return;
  }
  if (OP == OP_KEYPAIR) {
    msp::absorb_aligned<S, 168>(a, s, 0, v.coins + 32, 32, live);
  } else {
    uint2 kr[S::NS];
    msp::zero<S>(kr);
    if (OP == OP_ENC) {
      // m = SHA3-256(coins), H(pk), kr = SHA3-512(m || H(pk))  (cuda_kernel.cu:68-70)
      msp::absorb_aligned<S, 136>(kr, s, 0, v.coins, 32, live);
      msp::absorb_finish<S, 136>(kr, s, 32, 0x06u);
      msp::store<S>(kr, s, scr + Q::MTXT, 4, live);
      msp::keep<S>(kr, s, 4);  // lanes 0..3 = m
      const int pos = msp::absorb_aligned<S, 136>(a, s, 0, v.pk, P::PK, live);
      msp::absorb_finish<S, 136>(a, s, pos, 0x06u);
      msp::move4<S, 4>(kr, a, s);  // lanes 4..7 = H(pk)
    } else {
      // m' from the inner-product pass, H(pk) stored in sk (cuda_kernel.cu:231-232)
      const int pos = msp::absorb_aligned<S, 72>(kr, s, 0, scr + Q::MTXT, 32, live);
      msp::absorb_aligned<S, 72>(kr, s, pos, v.sk + P::SK - 64, 32, live);
    }
    msp::absorb_finish<S, 72>(kr, s, 64, 0x06u);
    msp::store<S>(kr, s, scr + Q::KR, 8, live);
    // GenSecret seed = kr[32:64] = lanes 4..7 -> lanes 0..3
    msp::zero<S>(a);
    msp::xor_lane<S, 0>(a, s, s.template get<4>(kr));
    msp::xor_lane<S, 1>(a, s, s.template get<5>(kr));
    msp::xor_lane<S, 2>(a, s, s.template get<6>(kr));
    msp::xor_lane<S, 3>(a, s, s.template get<7>(kr));
  }
  msp::absorb_finish<S, 168>(a, s, 32, 0x1Fu);
  msp::squeeze<S, 168>(a, s, scr + Q::SRAW, P::SRAW, live);
  if (OP == OP_DEC) {  // H(c) of the input ciphertext (see prologue_inst)
    msp::zero<S>(a);
    const int pos = msp::absorb_aligned<S, 136>(a, s, 0, v.ct, P::CT, live);
    msp::absorb_finish<S, 136>(a, s, pos, 0x06u);
    msp::store<S>(a, s, scr + Q::HC, 4, live);
  }
}

// Encaps finish: k = SHA3-256(kr[0:32] || SHA3-256(c)).
template <class S, int L>
__device__ __forceinline__ void finish_enc_multi(const Inst &v, const S &s, bool live) {
  using P = SP<L>;
  using Q = Scr<L>;
  uint2 h[S::NS], a[S::NS];
  msp::zero<S>(h);
  const int pos = msp::absorb_aligned<S, 136>(h, s, 0, v.ct, P::CT, live);
  msp::absorb_finish<S, 136>(h, s, pos, 0x06u);
  msp::zero<S>(a);
  msp::absorb_aligned<S, 136>(a, s, 0, v.scr + Q::KR, 32, live);
  msp::move4<S, 4>(a, h, s);
  msp::absorb_finish<S, 136>(a, s, 64, 0x06u);
  msp::store<S>(a, s, v.ss, 4, live);
}

// Keypair finish: sk = s || pk || H(pk) || z (the secret part was written by the product).
template <class S, int L>
__device__ __forceinline__ void finish_kp_multi(const Inst &v, const S &s, bool live) {
  using P = SP<L>;
  if (live && s.writer()) {
    const int t = s.lane(0) % 5;  // five threads share the copy (a warp per state: lanes 0..4)
    if (s.lane(0) < 5)
      for (int off = 8 * t; off < P::PK; off += 40)
        *reinterpret_cast<uint2 *>(v.sk + P::POLYVEC + off) = ld_lane(v.pk + off);
  }
  uint2 a[S::NS];
  msp::zero<S>(a);
  const int pos = msp::absorb_aligned<S, 136>(a, s, 0, v.pk, P::PK, live);
  msp::absorb_finish<S, 136>(a, s, pos, 0x06u);
  msp::store<S>(a, s, v.sk + P::SK - 64, 4, live);
  const int q = s.lane(0);
  if (live && s.writer() && q < 4) *reinterpret_cast<uint2 *>(v.sk + P::SK - 32 + 8 * q) = ld_lane(v.coins + 64 + 8 * q);
}

// ---------------------------------------------------------------- finish
template <int L, int OP>
__device__ __forceinline__ void finish_inst(const Inst &v) {
  using P = SP<L>;
  using S = Scr<L>;
  if (OP == OP_KEYPAIR) {
    const uint8_t *pk = v.pk;
    uint8_t *sk = v.sk;
    for (int off = 0; off < P::PK; off += 8) *reinterpret_cast<uint2 *>(sk + P::POLYVEC + off) = ld_lane(pk + off);
    uint2 h[4];
    sha3_256_msg(pk, P::PK, h);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      *reinterpret_cast<uint2 *>(sk + P::SK - 64 + 8 * q) = h[q];
      *reinterpret_cast<uint2 *>(sk + P::SK - 32 + 8 * q) = ld_lane(v.coins + 64 + 8 * q);
    }
    return;
  }
  const uint8_t *scr = v.scr;
  uint2 m[8], hc[4], k[4];
  if (OP == OP_DEC) {
#pragma unroll
    for (int q = 0; q < 4; q++) hc[q] = ld_lane(scr + S::HC + 8 * q);
  } else {
    sha3_256_msg(v.ct, P::CT, hc);
  }
  const uint32_t msk = OP == OP_DEC ? 0u - (uint32_t)(*v.fail != 0u) : 0u;
  const uint8_t *z = v.sk + P::SK - 32;
#pragma unroll
  for (int q = 0; q < 4; q++) {
    uint2 x = ld_lane(scr + S::KR + 8 * q);
    if (OP == OP_DEC) {  // cmov(kr, z, fail) before the final hash
      const uint2 y = ld_lane(z + 8 * q);
      x = make_uint2((x.x & ~msk) | (y.x & msk), (x.y & ~msk) | (y.y & msk));
    }
    m[q] = x;
    m[4 + q] = hc[q];
  }
  sha3_256_64(m, k);
#pragma unroll
  for (int q = 0; q < 4; q++) *reinterpret_cast<uint2 *>(v.ss + 8 * q) = k[q];
}

// ---------------------------------------------------------------- bit packing helpers
// Coefficient c of `bits` bits from a little-endian packed array in shared memory that is
// 4-byte aligned and readable 8 bytes past the coefficient: two aligned words, one funnel
// shift (sh <= 31 and sh + bits <= 44, so two words always suffice).
__device__ __forceinline__ uint32_t unpack_smem(const uint8_t *src, int c, int bits) {
  const int bit = c * bits, by = bit >> 3;
  const uint32_t *w = reinterpret_cast<const uint32_t *>(src + (by & ~3));
  return __funnelshift_r(w[0], w[1], (bit & 7) + 8 * (by & 3)) & ((1u << bits) - 1u);
}

// Unpacks NC little-endian BITS-bit fields from whole words (NC * BITS a multiple of 32)
// and calls f(i, value) for each; all bit offsets are compile-time after unrolling.
template <int BITS, int NC, class F>
__device__ __forceinline__ void unpack_words(const uint32_t *w, F &&f) {
  static_assert(NC * BITS % 32 == 0, "whole words");
  constexpr int NW = NC * BITS / 32;
  uint32_t r[NW + 1];
#pragma unroll
  for (int k = 0; k < NW; k++) r[k] = w[k];
  r[NW] = 0;
#pragma unroll
  for (int i = 0; i < NC; i++) {
    const int bit = i * BITS, k = bit >> 5, sh = bit & 31;
    const uint32_t v = sh + BITS <= 32 ? r[k] >> sh : __funnelshift_r(r[k], r[k + 1], sh);
    f(i, v & ((1u << BITS) - 1u));
  }
}

// Byte-wise two's-complement negation of four int8 lanes.
__device__ __forceinline__ uint32_t neg_bytes(uint32_t x) {
  return ((~x & 0x7F7F7F7Fu) + 0x01010101u) ^ (~x & 0x80808080u);
}

// Packs the G = 8 / gcd(BITS, 8) coefficients v[0..G) (each < 2^BITS) little-endian into
// G * BITS / 8 bytes at out: the smallest group that ends on a byte boundary, unrolled.
template <int BITS>
__device__ __forceinline__ constexpr int group_coefs() {
  return BITS % 8 == 0 ? 1 : BITS % 4 == 0 ? 2 : BITS % 2 == 0 ? 4 : 8;
}
template <int BITS>
__device__ __forceinline__ void pack_group(const uint16_t *v, uint8_t *out) {
  constexpr int G = group_coefs<BITS>();
  uint64_t acc = 0;
  int nb = 0, o = 0;
#pragma unroll
  for (int i = 0; i < G; i++) {
    acc |= (uint64_t)v[i] << nb;
    nb += BITS;
#pragma unroll
    for (int k = 0; k < 2; k++)
      if (nb >= 8) {
        out[o++] = (uint8_t)acc;
        acc >>= 8;
        nb -= 8;
      }
  }
}
// n coefficients (a multiple of the group size) into `out` (shared memory), CTA-wide.
// Group g on thread (off + g) mod blockDim: a second pack in the same phase starts where the
// first one's groups end.
template <int BITS>
__device__ __forceinline__ void pack_poly(const uint16_t *v, int n, uint8_t *out, int off = 0) {
  constexpr int G = group_coefs<BITS>(), NB = G * BITS / 8;
  const int nt = blockDim.x;
  for (int g = ((int)threadIdx.x + nt - off % nt) % nt; g < n / G; g += nt) pack_group<BITS>(v + g * G, out + g * NB);
}

__device__ __forceinline__ uint32_t pack_byte(const uint16_t *v, int q, int bits) {
  const int bit0 = 8 * q;
  int c = bit0 / bits;
  const int off = bit0 - c * bits;
  const uint32_t mask = (1u << bits) - 1u;
  uint32_t acc = (v[c] & mask) >> off;
  int have = bits - off;
  while (have < 8) {
    c++;
    acc |= (uint32_t)(v[c] & mask) << have;
    have += bits;
  }
  return acc & 0xFFu;
}

// ---------------------------------------------------------------- product kernel
// Shared-memory layout common to both forms.
template <int L>
struct PL {
  static constexpr int NO_MAX = L + 1;
  // Public polynomials are 264 u16 apart (528 B): polynomials read at the same offset
  // by neighbouring threads start 4 banks apart.
  static constexpr int PS = SN + 8;
  static constexpr int A16 = 0;                               // u16 [L*L][PS]
  static constexpr int B16 = A16 + L * L * PS * 2;            // u16 [L][PS] public b / b'
  static constexpr int SEC = B16 + L * PS * 2;                // s8  [L][256]
  static constexpr int RES = SEC + L * SN;                    // u16 [L+1][256]
  static constexpr int CM = RES + NO_MAX * SN * 2;            // u16 [256]
  static constexpr int SEQ = CM + SN * 2;                     // s8  [L][528] secret sequences
  static constexpr int SEQ_STRIDE = 528;
  static constexpr int COMMON = SEQ + L * SEQ_STRIDE;
  // tcgen05 form
  static constexpr int HANK = (COMMON + 127) & ~127;          // [L][62][128]
  static constexpr int HANK_STRIDE = 62 * 128;
  static constexpr int BOP = HANK + L * HANK_STRIDE;          // [NPAD/8][K/16][8][16]
  static constexpr int NPAD = 2 * NO_MAX <= 8 ? 8 : 16;
  static constexpr int BOP_GROUP = L * SN / 16 * 128;         // bytes per 8-row N group
  static constexpr int BAR = BOP + (NPAD / 8) * BOP_GROUP;
  static constexpr int TSLOT = BAR + 8;
  static constexpr int TC_TOTAL = TSLOT + 8;
  // Packed operands copied in from global memory before unpacking; the Hankel matrices
  // are built after the unpack, so the staging area reuses their space.  Each piece is
  // followed by 8 readable bytes (unpack_smem).
  static constexpr int ST_A = HANK;                                         // GenMatrix bytes
  static constexpr int ST_S = ST_A + SP<L>::ARAW + 8;                       // GenSecret bytes
  static constexpr int ST_P = ST_S + SP<L>::SRAW + 8;                       // packed b (pk)
  static constexpr int ST_END = ST_P + SP<L>::POLYVECCOMP + 8;
  static constexpr int ST_SK = HANK;                                        // decaps inner: 13-bit s
  static constexpr int ST_CT = ST_SK + SP<L>::POLYVEC + 8;                  // and the ciphertext
  static constexpr int ST_END_INNER = ST_CT + SP<L>::CT + 8;
  static constexpr int DP4A_TOTAL = ST_END > ST_END_INNER ? ST_END : ST_END_INNER;
};

template <int L, int MODE>
__device__ __forceinline__ constexpr int n_out() {
  return MODE == PM_KEYPAIR ? L : MODE == PM_DEC_INNER ? 1 : L + 1;
}

// 8-byte copy of `bytes` (a multiple of 8, both ends 8-byte aligned) by the whole CTA.
__device__ __forceinline__ void copy8(uint8_t *dst, const uint8_t *src, int bytes) {
  for (int q = threadIdx.x; q < bytes / 8; q += blockDim.x)
    reinterpret_cast<uint2 *>(dst)[q] = reinterpret_cast<const uint2 *>(src)[q];
}

// Phase 1: secrets and public polynomials into shared memory.  The packed inputs are
// first copied in with 8-byte loads (a handful per thread), then unpacked from shared
// memory, instead of up to three byte loads from global memory per coefficient.
// The packed inputs of one instance as 8-byte words: source in global memory and
// destination in the staging area.
template <int L, int MODE>
struct Staged {
  using P = SP<L>;
  using Y = PL<L>;
  static_assert(P::ARAW % 8 == 0 && P::SRAW % 8 == 0 && P::POLYVECCOMP % 8 == 0 && P::POLYVEC % 8 == 0 &&
                    P::CT % 8 == 0,
                "8-byte staging");
  static constexpr bool INNER = MODE == PM_DEC_INNER;
  static constexpr int W0 = (INNER ? P::POLYVEC : P::ARAW) / 8;                      // words of piece 0
  static constexpr int W1 = (INNER ? P::CT : P::SRAW) / 8;                            // piece 1
  static constexpr int W2 = (INNER || MODE == PM_KEYPAIR) ? 0 : P::POLYVECCOMP / 8;  // piece 2
  // piece 3: the message bits m (32 bytes of scratch) that the epilogue encodes into v'
  // (encaps, decaps re-encryption), staged in the CM region, which only the inner pass uses
  static constexpr int W3 = (INNER || MODE == PM_KEYPAIR) ? 0 : 4;
  static constexpr int WORDS = W0 + W1 + W2 + W3;
  static constexpr int PER_THREAD = (WORDS + 255) / 256;  // with 256 threads
  __device__ __forceinline__ static const uint2 *src(const Inst &v, int w) {
    if (INNER)
      return w < W0 ? reinterpret_cast<const uint2 *>(v.sk) + w : reinterpret_cast<const uint2 *>(v.ct) + (w - W0);
    if (w < W0) return reinterpret_cast<const uint2 *>(v.scr + Scr<L>::ARAW) + w;
    if (w < W0 + W1) return reinterpret_cast<const uint2 *>(v.scr + Scr<L>::SRAW) + (w - W0);
    if (w < W0 + W1 + W2)
      return reinterpret_cast<const uint2 *>(MODE == PM_ENC ? v.pk : v.sk + P::POLYVEC) + (w - W0 - W1);
    return reinterpret_cast<const uint2 *>(v.scr + Scr<L>::MTXT) + (w - W0 - W1 - W2);
  }
  __device__ __forceinline__ static uint2 *dst(uint8_t *sm, int w) {
    if (INNER)
      return w < W0 ? reinterpret_cast<uint2 *>(sm + Y::ST_SK) + w : reinterpret_cast<uint2 *>(sm + Y::ST_CT) + (w - W0);
    if (w < W0) return reinterpret_cast<uint2 *>(sm + Y::ST_A) + w;
    if (w < W0 + W1) return reinterpret_cast<uint2 *>(sm + Y::ST_S) + (w - W0);
    if (w < W0 + W1 + W2) return reinterpret_cast<uint2 *>(sm + Y::ST_P) + (w - W0 - W1);
    return reinterpret_cast<uint2 *>(sm + Y::CM) + (w - W0 - W1 - W2);
  }
};

// Copy one instance's packed inputs into the staging area (CTA-wide, 8-byte accesses).
template <int L, int MODE>
__device__ __forceinline__ void stage_operands(const Inst &v, uint8_t *sm) {
  using T = Staged<L, MODE>;
  for (int w = threadIdx.x; w < T::WORDS; w += blockDim.x) *T::dst(sm, w) = *T::src(v, w);
}

// The same copy split in two for a persistent loop (256 threads): load() into registers
// early, store() into the staging area once it is free.
template <int L, int MODE>
struct OperandPrefetch {
  using T = Staged<L, MODE>;
  uint2 r[T::PER_THREAD];
  __device__ __forceinline__ void load(const Inst &v) {
#pragma unroll
    for (int k = 0; k < T::PER_THREAD; k++) {
      const int w = threadIdx.x + 256 * k;
      if (w < T::WORDS) r[k] = *T::src(v, w);
    }
  }
  __device__ __forceinline__ void store(uint8_t *sm) const {
#pragma unroll
    for (int k = 0; k < T::PER_THREAD; k++) {
      const int w = threadIdx.x + 256 * k;
      if (w < T::WORDS) *T::dst(sm, w) = r[k];
    }
  }
};

template <int L, int MODE>
__device__ __forceinline__ void unpack_operands(const Inst &v, uint8_t *sm);

template <int L, int MODE>
__device__ __forceinline__ void load_operands(const Inst &v, uint8_t *sm) {
  stage_operands<L, MODE>(v, sm);
  __syncthreads();
  unpack_operands<L, MODE>(v, sm);
}

// Unpack the staged inputs (after stage_operands or a prefetch's store, and a CTA barrier).
template <int L, int MODE>
__device__ __forceinline__ void unpack_operands(const Inst &v, uint8_t *sm) {
  using P = SP<L>;
  using Y = PL<L>;
  static_assert(Y::DP4A_TOTAL <= Y::TC_TOTAL, "staging must fit the tensor form's layout");
  const int tid = threadIdx.x;
  uint32_t *secw = reinterpret_cast<uint32_t *>(sm + Y::SEC);  // 4 int8 coefficients per word
  uint16_t *a16 = reinterpret_cast<uint16_t *>(sm + Y::A16);
  uint16_t *b16 = reinterpret_cast<uint16_t *>(sm + Y::B16);
  uint16_t *cm = reinterpret_cast<uint16_t *>(sm + Y::CM);
  // Public polynomials with 10-bit coefficients: 16 coefficients (5 words) per thread, two
  // 16-byte stores.
  // The unpack loops of one mode start at disjoint thread ranges (job g of a loop that starts
  // at thread `off` runs on thread off + g), so no thread does two jobs while others wait at
  // the barrier that follows: l = 3 encaps has 48 + 72 + 48 jobs for 256 threads.
  auto job0 = [&](int off) { return (tid + (int)blockDim.x - off) % (int)blockDim.x; };
  auto unpack_p = [&](const uint8_t *src, int off) {
    for (int g = job0(off); g < L * SN / 16; g += blockDim.x) {
      uint32_t o[8];
      unpack_words<EP, 16>(reinterpret_cast<const uint32_t *>(src) + 5 * g, [&](int i, uint32_t x) {
        if (i & 1) o[i >> 1] |= x << 16;
        else o[i >> 1] = x;
      });
      uint4 *d = reinterpret_cast<uint4 *>(b16 + (g >> 4) * Y::PS + 16 * (g & 15));
      d[0] = make_uint4(o[0], o[1], o[2], o[3]);
      d[1] = make_uint4(o[4], o[5], o[6], o[7]);
    }
  };
  if (MODE == PM_DEC_INNER) {
    const uint8_t *ct = sm + Y::ST_CT;
    // 13-bit secret from sk, centred: 32 coefficients (13 words) per thread.
    for (int g = tid; g < L * SN / 32; g += blockDim.x) {
      uint32_t o[8];
      unpack_words<EQ, 32>(reinterpret_cast<const uint32_t *>(sm + Y::ST_SK) + 13 * g, [&](int i, uint32_t x) {
        const uint32_t b = x & 0xFFu;  // low byte of the centred value (|s| < 128)
        if ((i & 3) == 0) o[i >> 2] = b;
        else o[i >> 2] |= b << (8 * (i & 3));
      });
      uint4 *d = reinterpret_cast<uint4 *>(secw + 8 * g);
      d[0] = make_uint4(o[0], o[1], o[2], o[3]);
      d[1] = make_uint4(o[4], o[5], o[6], o[7]);
    }
    unpack_p(ct, L * SN / 32);
    for (int c = tid; c < SN; c += blockDim.x) cm[c] = (uint16_t)unpack_smem(ct + P::POLYVECCOMP, c, P::ET);
  } else {
    // CBD_mu from the GenSecret bytes: 16 coefficients (mu/2 words) per thread.
    constexpr uint32_t hm = (1u << (P::MU / 2)) - 1u;
    for (int g = job0(0); g < L * SN / 16; g += blockDim.x) {
      uint32_t o[4];
      unpack_words<P::MU, 16>(reinterpret_cast<const uint32_t *>(sm + Y::ST_S) + (P::MU / 2) * g,
                              [&](int i, uint32_t x) {
                                const uint32_t b = (uint32_t)(__popc(x & hm) - __popc((x >> (P::MU / 2)) & hm)) & 0xFFu;
                                if ((i & 3) == 0) o[i >> 2] = b;
                                else o[i >> 2] |= b << (8 * (i & 3));
                              });
      reinterpret_cast<uint4 *>(secw)[g] = make_uint4(o[0], o[1], o[2], o[3]);
    }
    // GenMatrix: 13-bit coefficients, 32 (13 words) per thread, four 16-byte stores.
    for (int g = job0(L * SN / 16); g < L * L * SN / 32; g += blockDim.x) {
      uint32_t o[16];
      unpack_words<EQ, 32>(reinterpret_cast<const uint32_t *>(sm + Y::ST_A) + 13 * g, [&](int i, uint32_t x) {
        if (i & 1) o[i >> 1] |= x << 16;
        else o[i >> 1] = x;
      });
      uint4 *d = reinterpret_cast<uint4 *>(a16 + (g >> 3) * Y::PS + 32 * (g & 7));
#pragma unroll
      for (int q = 0; q < 4; q++) d[q] = make_uint4(o[4 * q], o[4 * q + 1], o[4 * q + 2], o[4 * q + 3]);
    }
    if (MODE != PM_KEYPAIR) unpack_p(sm + Y::ST_P, L * SN / 16 + L * L * SN / 32);
  }
}

// Secret sequences, one 32-bit word (4 int8) per thread step, from the secrets in SEC.
//   TC  : E_j[e] = s_ext[e - 255], e in [0, 528): -s[e + 1] for e < 255, s[e - 255] for
//         255 <= e < 511, 0 above (the Hankel generating sequence).
//   dp4a: R_j[t] = s_ext[255 - t]: s[255 - t] for t < 256, -s[511 - t] below 512, 0 above.
template <int L, bool TC>
__device__ __forceinline__ void build_seq(uint8_t *sm) {
  using Y = PL<L>;
  constexpr int NW = Y::SEQ_STRIDE / 4;  // 132
  const uint32_t *secw = reinterpret_cast<const uint32_t *>(sm + Y::SEC);
  uint32_t *seqw = reinterpret_cast<uint32_t *>(sm + Y::SEQ);
  for (int x = threadIdx.x; x < L * NW; x += blockDim.x) {
    const int j = x / NW, k = x - j * NW;
    const uint32_t *sw = secw + 64 * j;
    uint32_t e = 0;
    if (TC) {
      if (k <= 63) e = neg_bytes(__funnelshift_r(sw[k], k < 63 ? sw[k + 1] : 0u, 8));
      else if (k <= 127) e = __funnelshift_r(sw[k - 64], k < 127 ? sw[k - 63] : 0u, 8);
      if (k == 63) e |= sw[0] << 24;
    } else {
      if (k < 64) e = __byte_perm(sw[63 - k], 0, 0x0123);
      else if (k < 128) e = neg_bytes(__byte_perm(sw[127 - k], 0, 0x0123));
    }
    seqw[x] = e;
  }
}

// Public polynomial multiplied by secret j for output o.
template <int L, int MODE>
__device__ __forceinline__ const uint16_t *pub_poly(const uint8_t *sm, int o, int j) {
  using Y = PL<L>;
  const uint16_t *a16 = reinterpret_cast<const uint16_t *>(sm + Y::A16);
  const uint16_t *b16 = reinterpret_cast<const uint16_t *>(sm + Y::B16);
  if (MODE == PM_DEC_INNER) return b16 + j * Y::PS;
  if (MODE == PM_KEYPAIR) return a16 + (j * L + o) * Y::PS;  // transposed: b = A^T s
  return o < L ? a16 + (o * L + j) * Y::PS : b16 + j * Y::PS;
}

// Phase 3: rounding, packing / comparison.  res holds the products mod 2^16.
template <int L, int MODE>
__device__ __forceinline__ void epilogue(const Inst &v, uint8_t *sm) {
  using P = SP<L>;
  using S = Scr<L>;
  using Y = PL<L>;
  const int tid = threadIdx.x, nt = blockDim.x;
  uint16_t *res = reinterpret_cast<uint16_t *>(sm + Y::RES);
  uint8_t *scr = v.scr;
  if (MODE == PM_DEC_INNER) {
    const uint16_t *cm = reinterpret_cast<const uint16_t *>(sm + Y::CM);
    for (int c = tid; c < SN; c += nt)
      res[c] = (uint16_t)(((uint32_t)res[c] + P::H2 - ((uint32_t)cm[c] << (EP - P::ET))) >> (EP - 1)) & 1u;
    __syncthreads();
    if (tid < 32) scr[S::MTXT + tid] = (uint8_t)pack_byte(res, tid, 1);
    return;
  }
  for (int c = tid; c < L * SN; c += nt) res[c] = (uint16_t)((((uint32_t)res[c] + P::H1) >> (EQ - EP)) & 0x3FFu);
  if (MODE != PM_KEYPAIR) {
    const uint8_t *mt = sm + Y::CM;  // staged with the operands
    for (int c = tid; c < SN; c += nt) {
      const uint32_t mb = (mt[c >> 3] >> (c & 7)) & 1u;
      res[L * SN + c] = (uint16_t)((((uint32_t)res[L * SN + c] - (mb << (EP - 1)) + P::H1) >> (EP - P::ET)) &
                                   ((1u << P::ET) - 1u));
    }
  }
  __syncthreads();
  // Pack into shared memory (the staging area, free again), then 8-byte stores / compares.
  uint8_t *stg = sm + Y::ST_A;
  if (MODE == PM_KEYPAIR) {
    const int8_t *sec = reinterpret_cast<const int8_t *>(sm + Y::SEC);
    pack_poly<EP>(res, L * SN, stg);  // POLYVECCOMP bytes
    uint16_t *s13 = reinterpret_cast<uint16_t *>(sm + Y::A16);  // A no longer needed
    for (int c = tid; c < L * SN; c += nt) s13[c] = (uint16_t)((int32_t)sec[c] & 0x1FFF);
    __syncthreads();
    pack_poly<EQ>(s13, L * SN, stg + P::POLYVECCOMP);  // POLYVEC bytes
    __syncthreads();
    copy8(v.pk, stg, P::POLYVECCOMP);
    copy8(v.sk, stg + P::POLYVECCOMP, P::POLYVEC);
    return;
  }
  pack_poly<EP>(res, L * SN, stg);
  pack_poly<P::ET>(res + L * SN, SN, stg + P::POLYVECCOMP, L * SN / group_coefs<EP>());
  __syncthreads();
  if (MODE == PM_ENC) {
    copy8(v.ct, stg, P::CT);
  } else {
    uint32_t diff = 0;
    for (int q = tid; q < P::CT / 8; q += nt) {
      const uint2 a = reinterpret_cast<const uint2 *>(stg)[q], b = reinterpret_cast<const uint2 *>(v.ct)[q];
      diff |= (a.x ^ b.x) | (a.y ^ b.y);
    }
    const int any = __syncthreads_or(diff != 0);
    if (tid == 0) *v.fail = (uint32_t)any;
  }
}

// ---------------------------------------------------------------- dp4a form
// Secret j's reversed sign-extended window R_j[t] = s_ext[255 - t], t in [0, 512), with
// s_ext[d] = s[d] (d >= 0), -s[d + 256] (d < 0): coefficient i of s*P is
// sum_m P[m] R_j[255 - i + m].
// I32 = true is the INT32 schoolbook form (SABER-GPU/src/poly.cu:209-358, the reference's
// mode 1): the same window, one 32-bit multiply-add per coefficient pair instead of dp2a.
template <int L, int MODE, bool I32 = false>
__device__ __forceinline__ void product_dp4a_cta(const Inst &v, uint8_t *sm) {
  using Y = PL<L>;
  constexpr int NO = n_out<L, MODE>();
  const int tid = threadIdx.x;
  load_operands<L, MODE>(v, sm);
  __syncthreads();
  build_seq<L, false>(sm);
  __syncthreads();
  const int base = 255 - tid, wb = base >> 2, sh = 8 * (base & 3);
  int acc[NO];
#pragma unroll
  for (int o = 0; o < NO; o++) acc[o] = 0;
  for (int j = 0; j < L; j++) {
    const uint32_t *rw = reinterpret_cast<const uint32_t *>(sm + Y::SEQ + j * Y::SEQ_STRIDE);
    const uint2 *pp[NO];
#pragma unroll
    for (int o = 0; o < NO; o++) pp[o] = reinterpret_cast<const uint2 *>(pub_poly<L, MODE>(sm, o, j));
    uint32_t w0 = rw[wb];
#pragma unroll 4
    for (int mq = 0; mq < SN / 4; mq++) {
      const uint32_t w1 = rw[wb + mq + 1];
      const int win = (int)__funnelshift_r(w0, w1, sh);
      w0 = w1;
      if (I32) {
        const int s0 = (int)(int8_t)win, s1 = (int)(int8_t)(win >> 8), s2 = (int)(int8_t)(win >> 16),
                  s3 = win >> 24;
#pragma unroll
        for (int o = 0; o < NO; o++) {
          const uint2 pw = pp[o][mq];
          acc[o] += (int)(pw.x & 0xFFFFu) * s0 + (int)(pw.x >> 16) * s1 + (int)(pw.y & 0xFFFFu) * s2 +
                    (int)(pw.y >> 16) * s3;
        }
      } else {
#pragma unroll
        for (int o = 0; o < NO; o++) {
          const uint2 pw = pp[o][mq];
          acc[o] = dp2a_hi((int)pw.y, win, dp2a_lo((int)pw.x, win, acc[o]));
        }
      }
    }
  }
  uint16_t *res = reinterpret_cast<uint16_t *>(sm + Y::RES);
#pragma unroll
  for (int o = 0; o < NO; o++) res[o * SN + tid] = (uint16_t)acc[o];
  __syncthreads();
  epilogue<L, MODE>(v, sm);
  __syncthreads();
}

// ---------------------------------------------------------------- tcgen05 form
// TMEM columns [tbase, tbase + 32) must be allocated by the caller; the mbarrier in
// shared memory is initialised here.  Returns false if the bounded wait expired.
// From unpacked operands to the stored result: secret sequences, Hankel and B operand
// tiles, the MMAs (completion on the mbarrier at Y::BAR, parity `phase`), the TMEM
// read-back and the epilogue.  Returns false if the bounded wait expired.
template <int L, int MODE>
__device__ __forceinline__ bool tc_mma_epilogue(const Inst &v, uint8_t *sm, uint32_t tbase, uint32_t *err,
                                                uint32_t phase);

template <int L, int MODE>
__device__ __forceinline__ bool product_tc_cta(const Inst &v, uint8_t *sm, uint32_t tbase, uint32_t *err) {
  using Y = PL<L>;
  uint64_t *bar = reinterpret_cast<uint64_t *>(sm + Y::BAR);
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  load_operands<L, MODE>(v, sm);
  __syncthreads();
  const bool ok = tc_mma_epilogue<L, MODE>(v, sm, tbase, err, 0);
  if (threadIdx.x == 0 && ok) mbar_inval(bar);
  return ok;
}

template <int L, int MODE>
__device__ __forceinline__ bool tc_mma_epilogue(const Inst &v, uint8_t *sm, uint32_t tbase, uint32_t *err,
                                                uint32_t phase) {
  using Y = PL<L>;
  constexpr int NO = n_out<L, MODE>();
  constexpr int NPAD = 2 * NO <= 8 ? 8 : 16;
  uint64_t *bar = reinterpret_cast<uint64_t *>(sm + Y::BAR);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  build_seq<L, true>(sm);
  __syncthreads();
  // Hankel core matrices: H_j[t][r][c] = E_j[8t + r + c].  Row r = tid % 8 is fixed per
  // thread; (j, t) advance by 32 core matrices per step, and 8 consecutive threads write one
  // 128-byte core matrix.
  {
    const int r = tid & 7, sh = 8 * (r & 3);
    int j = 0, t = tid >> 3;
    while (j < L) {
      const uint32_t *sw = reinterpret_cast<const uint32_t *>(sm + Y::SEQ + j * Y::SEQ_STRIDE) + 2 * t + (r >> 2);
      const uint32_t x0 = sw[0], x1 = sw[1], x2 = sw[2], x3 = sw[3], x4 = sw[4];
      *reinterpret_cast<uint4 *>(sm + Y::HANK + j * Y::HANK_STRIDE + t * 128 + r * 16) =
          make_uint4(__funnelshift_r(x0, x1, sh), __funnelshift_r(x1, x2, sh), __funnelshift_r(x2, x3, sh),
                     __funnelshift_r(x3, x4, sh));
      t += 32;
      if (t >= 62) {
        t -= 62;
        j++;
      }
    }
  }
  // B operand: row n = o + NO*limb, K = 256 j + k', value = limb(P_{o,j}[255 - k']).  One
  // thread per (row n, 16-column chunk kc): coefficients 255-k0 .. 240-k0 are two aligned
  // 16-byte reads (8 little-endian pairs); a PRMT turns two pairs into 4 output bytes,
  // reversed.  Threads n = 0..7 of a chunk write its 128 bytes contiguously.
  for (int x = tid; x < NPAD * L * (SN / 16); x += 256) {
    const int n = (x & 7) + 8 * (x / (8 * L * (SN / 16))), kc = (x >> 3) % (L * SN / 16);
    const int j = kc / (SN / 16), k0 = 16 * (kc % (SN / 16));
    uint4 out = make_uint4(0, 0, 0, 0);
    if (n < 2 * NO) {
      const int o = n % NO;
      const uint32_t sel = n < NO ? 0x4602u : 0x5713u;  // low / high byte of each coefficient
      const uint4 *pw = reinterpret_cast<const uint4 *>(pub_poly<L, MODE>(sm, o, j) + 240 - k0);
      const uint4 w0 = pw[0], w1 = pw[1];  // coefficients 240-k0 .. 247-k0 and 248-k0 .. 255-k0
      out = make_uint4(prmt(w1.w, w1.z, sel), prmt(w1.y, w1.x, sel), prmt(w0.w, w0.z, sel), prmt(w0.y, w0.x, sel));
    }
    *reinterpret_cast<uint4 *>(sm + Y::BOP + (n >> 3) * Y::BOP_GROUP + kc * 128 + (n & 7) * 16) = out;
  }
  fence_proxy_async_smem();
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (tid == 0) {
    constexpr uint32_t idesc = idesc_i8(128, NPAD, true, false, false, false);
    // Base descriptors; a step moves only the start-address field (address / 16, low word).
    const uint64_t a0 = sdesc(smem_u32(sm + Y::HANK), 256, 128), b0 = sdesc(smem_u32(sm + Y::BOP), 128, Y::BOP_GROUP);
#pragma unroll
    for (int mt = 0; mt < 2; mt++)
#pragma unroll
      for (int j = 0; j < L; j++)
#pragma unroll
        for (int ks = 0; ks < 8; ks++)
          mma_i8(tbase + mt * NPAD, a0 + (uint64_t)((j * Y::HANK_STRIDE + (16 * mt + 4 * ks) * 128) >> 4),
                 b0 + (uint64_t)(((16 * j + 2 * ks) * 128) >> 4), idesc, (j | ks) ? 1u : 0u);
    mma_commit(bar);
  }
  const bool ok = mbar_wait(bar, phase);
  if (!ok && lane == 0) atomicOr(err, DEV_ERR_TIMEOUT);
  tc_fence_after();
  // Warp w reads TMEM lanes 32 (w % 4) .. of M tile w / 4: coefficient = tid.
  uint32_t r[16];
  tmem_ld16(tbase + ((uint32_t)((warp & 3) * 32) << 16) + (warp >> 2) * NPAD, r);
  tmem_wait_ld();
  uint16_t *res = reinterpret_cast<uint16_t *>(sm + Y::RES);
#pragma unroll
  for (int o = 0; o < NO; o++) res[o * SN + tid] = (uint16_t)(r[o] + (r[NO + o] << 8));
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  epilogue<L, MODE>(v, sm);
  __syncthreads();
  return ok;
}

}  // namespace sdev
}  // namespace dpkem
