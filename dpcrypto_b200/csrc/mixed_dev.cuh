// Device side of the persistent mixed-scheme kernels (mixed.cu: one launch over a planned
// task list; serve.cu: a long-lived service fed from a host-written request ring): stage
// codes and kinds, per-request scratch records, the request record the kernels read, and
// the stage bodies (one instance per thread, a warp per instance, or a CTA per instance)
// built from the routines the batched kernels use.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>

#include "coins_dev.cuh"
#include "frodo_dev.cuh"
#include "saber_dev.cuh"

namespace dpkem {
namespace mixed {

// ---- stage codes: scheme * 128 + op * 32 + stage * 4 + form ----
__host__ __device__ constexpr int code_of(int scheme, int op, int stage, int form) {
  return scheme * 128 + op * 32 + stage * 4 + form;
}
__host__ __device__ constexpr int scheme_of(int code) { return code >> 7; }
__host__ __device__ constexpr int op_of(int code) { return (code >> 5) & 3; }
__host__ __device__ constexpr int stage_of(int code) { return (code >> 2) & 7; }
__host__ __device__ constexpr int form_of(int code) { return code & 3; }

// Stage kinds: 0 = thread (one instance per thread), 2 = thread with two roles (instance
// t on threads t and t + 128: Saber's two prologue sponges, Frodo decaps' prologue and
// ciphertext pre-absorb), 1 = CTA (one instance per task).
enum Kind : int { K_THREAD = 0, K_CTA = 1, K_THREAD2 = 2 };

// Task code flag (above the stage code's 10 bits, masked off before decoding): a
// thread-level stage run on a warp per instance (and role): the Keccak
// sponges spread over the warp's lanes (keccak25.cuh), 8 instances per task (4 for two-role
// stages).  The planner uses it for groups small enough that one thread per instance would
// leave the GPU idle (knob mixed_warp_max).
constexpr int kWarpTask = 1 << 10;
static_assert(code_of(4, 3, 7, 3) < kWarpTask, "stage codes must stay below the warp-task flag");

__host__ __device__ constexpr int nstages(int scheme, int op) { return op == OP_DEC ? 4 : 3; }

__host__ __device__ constexpr int kind_of(int scheme, int op, int stage) {
  if (scheme <= 1) {  // FrodoKEM-976, SHAKE (0) or AES (1)
    if (op == OP_DEC) return stage == 0 || stage == 2 ? K_CTA : stage == 1 ? K_THREAD2 : K_THREAD;
    return stage == 1 ? K_CTA : K_THREAD;
  }
  if (op == OP_DEC) return stage == 1 ? K_THREAD2 : stage == 3 ? K_THREAD : K_CTA;
  return stage == 0 ? K_THREAD2 : stage == 1 ? K_CTA : K_THREAD;
}

// Completed-role count an instance must show before `stage` may start.
__host__ __device__ constexpr uint32_t threshold(int scheme, int op, int stage) {
  uint32_t t = 0;
  for (int s = 0; s < stage; s++) t += kind_of(scheme, op, s) == K_THREAD2 ? 2u : 1u;
  return t;
}

// ---- per-request scratch records (256-byte multiples so no line is shared) ----
constexpr size_t kFrodoRec = 31744;  // rw 31,360 | k 24 | mu 24 | fail 4 (+12) | sponge 200
constexpr size_t kFrodoK = frodo::RW * 2, kFrodoMu = kFrodoK + 24, kFrodoFail = kFrodoMu + 24;
constexpr size_t kFrodoHs = kFrodoFail + 16;
constexpr size_t kFrodoCoins = kFrodoHs + 200;  // 64 B of device-drawn coins
static_assert(kFrodoCoins + 64 <= kFrodoRec, "Frodo record too small");

// Saber record: scratch | fail word | two 96-byte coin slots (one per prologue role).
__host__ __device__ inline size_t saber_scr_bytes(int level) {
  return level == 2 ? sdev::Scr<2>::BYTES : level == 3 ? sdev::Scr<3>::BYTES : sdev::Scr<4>::BYTES;
}
__host__ __device__ inline size_t saber_coins_off(int level) { return (saber_scr_bytes(level) + 4 + 7) & ~(size_t)7; }
__host__ __device__ inline size_t saber_rec_bytes(int level) {
  return (saber_coins_off(level) + 192 + 255) & ~(size_t)255;
}

struct DevReq {
  int32_t scheme, op;
  const uint8_t *in0, *in1;
  uint8_t *out0, *out1;
  uint8_t *scr;
  uint64_t coin_index;  // with gen: coins = SHAKE256(key || LE64(coin_index) || tag), drawn into in0
  uint32_t gen;
  uint32_t ticket;  // service requests: the ticket whose completion the last stage reports
};

// Draws a request's coins into `dst` (the first stage of a keypair / encaps whose request
// carried none): tag "kp" / "enc", length of the scheme's coins.
__device__ __forceinline__ void draw_coins(const CoinKey &key, const DevReq &r, uint8_t *dst) {
  const uint8_t kp[2] = {'k', 'p'}, enc[3] = {'e', 'n', 'c'};
  const bool is_kp = r.op == OP_KEYPAIR;
  const int len = r.scheme <= 1 ? (is_kp ? frodo::KP_COINS : frodo::ENC_COINS) : (is_kp ? 96 : 32);
  coin_generate(key, r.coin_index, is_kp ? kp : enc, is_kp ? 2 : 3, len, dst);
}

__device__ __forceinline__ fdev::Inst frodo_view(const DevReq &r) {
  fdev::Inst v{};
  const bool kp = r.op == OP_KEYPAIR, enc = r.op == OP_ENC;
  v.coins = kp || enc ? r.in0 : nullptr;
  v.pk = kp ? r.out0 : enc ? const_cast<uint8_t *>(r.in1) : nullptr;
  v.sk = kp ? r.out1 : enc ? nullptr : const_cast<uint8_t *>(r.in1);
  v.ct = enc ? r.out0 : kp ? nullptr : const_cast<uint8_t *>(r.in0);
  v.ss = enc ? r.out1 : kp ? nullptr : r.out0;
  v.rw = reinterpret_cast<uint16_t *>(r.scr);
  v.kk = r.scr + kFrodoK;
  v.mu = r.scr + kFrodoMu;
  v.fail = reinterpret_cast<uint32_t *>(r.scr + kFrodoFail);
  v.hs = reinterpret_cast<uint2 *>(r.scr + kFrodoHs);
  return v;
}

template <int L>
__device__ __forceinline__ sdev::Inst saber_view(const DevReq &r) {
  sdev::Inst v{};
  const bool kp = r.op == OP_KEYPAIR, enc = r.op == OP_ENC;
  v.coins = kp || enc ? r.in0 : nullptr;
  v.pk = kp ? r.out0 : enc ? const_cast<uint8_t *>(r.in1) : nullptr;
  v.sk = kp ? r.out1 : enc ? nullptr : const_cast<uint8_t *>(r.in1);
  v.ct = enc ? r.out0 : kp ? nullptr : const_cast<uint8_t *>(r.in0);
  v.ss = enc ? r.out1 : kp ? nullptr : r.out0;
  v.scr = r.scr;
  v.fail = reinterpret_cast<uint32_t *>(r.scr + sdev::Scr<L>::BYTES);
  return v;
}

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Spin loads: a relaxed load reads L2 (these kernels bypass L1) without the L1 invalidation
// an acquire load performs on every iteration, which would evict the register spills of the
// CTA sharing the SM; a spin that succeeds then fences once (__threadfence), which orders
// the loads after it behind the value it saw.
__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}


template <int L>
__device__ __forceinline__ void saber_thread(const CoinKey &key, int op, int stage, const DevReq &r, int role) {
  sdev::Inst v = saber_view<L>(r);
  if (r.gen && stage == 0 && op != OP_DEC) {
    // each prologue role draws its own copy (role 1 into the second slot), so neither
    // waits for the other; later stages read the first slot through in0
    uint8_t *slot = const_cast<uint8_t *>(r.in0) + (role ? 96 : 0);
    if (role == 0 || op == OP_KEYPAIR) draw_coins(key, r, slot);
    v.coins = slot;
  }
  if (op == OP_KEYPAIR) {
    if (stage == 0) sdev::prologue_inst<L, OP_KEYPAIR>(v, role);
    else sdev::finish_inst<L, OP_KEYPAIR>(v);
  } else if (op == OP_ENC) {
    if (stage == 0) sdev::prologue_inst<L, OP_ENC>(v, role);
    else sdev::finish_inst<L, OP_ENC>(v);
  } else {
    if (stage == 1) sdev::prologue_inst<L, OP_DEC>(v, role);
    else sdev::finish_inst<L, OP_DEC>(v);
  }
}

// The same stages on a warp per instance (a warp-wide call: every lane runs it).
template <int L>
__device__ __forceinline__ void saber_warp(const CoinKey &key, int op, int stage, const DevReq &r, int role) {
  using S = msp::Multi<1>;
  const S s(nullptr);
  sdev::Inst v = saber_view<L>(r);
  if (r.gen && stage == 0 && op != OP_DEC) {
    uint8_t *slot = const_cast<uint8_t *>(r.in0) + (role ? 96 : 0);
    if ((role == 0 || op == OP_KEYPAIR) && (threadIdx.x & 31) == 0) draw_coins(key, r, slot);
    __syncwarp();
    v.coins = slot;
  }
  if (op == OP_KEYPAIR) {
    if (stage == 0) sdev::prologue_multi<S, L, OP_KEYPAIR>(v, s, role, true);
    else sdev::finish_kp_multi<S, L>(v, s, true);
  } else if (op == OP_ENC) {
    if (stage == 0) sdev::prologue_multi<S, L, OP_ENC>(v, s, role, true);
    else sdev::finish_enc_multi<S, L>(v, s, true);
  } else {
    if (stage == 1) sdev::prologue_multi<S, L, OP_DEC>(v, s, role, true);
    else if ((threadIdx.x & 31) == 0) sdev::finish_inst<L, OP_DEC>(v);  // one permutation
  }
}

__device__ __forceinline__ void warp_stage(const CoinKey &key, int code, const DevReq &r, int role) {
  using S = msp::Multi<1>;
  const int scheme = scheme_of(code), op = op_of(code), stage = stage_of(code);
  if (scheme <= 1) {
    if (r.gen && stage == 0 && op != OP_DEC) {
      if ((threadIdx.x & 31) == 0) draw_coins(key, r, const_cast<uint8_t *>(r.in0));
      __syncwarp();
    }
    const S s(nullptr);
    const fdev::Inst v = frodo_view(r);
    if (op == OP_KEYPAIR) {
      if (stage == 0) fdev::kp_prologue_multi<S>(v, s, true);
      else fdev::pk_hash_multi<S>(v, s, true);
    } else if (op == OP_ENC) {
      if (stage == 0) fdev::prologue_multi<S, OP_ENC>(v, s, true);
      else fdev::ss_multi<S, OP_ENC>(v, s, true);
    } else {
      if (stage == 1 && role == 0) fdev::prologue_multi<S, OP_DEC>(v, s, true);
      else if (stage == 1) fdev::ct_absorb_multi<S>(v, s, true);
      else fdev::ss_multi<S, OP_DEC>(v, s, true);
    }
  } else if (scheme == 2) {
    saber_warp<2>(key, op, stage, r, role);
  } else if (scheme == 3) {
    saber_warp<3>(key, op, stage, r, role);
  } else {
    saber_warp<4>(key, op, stage, r, role);
  }
}

__device__ __forceinline__ void thread_stage(const CoinKey &key, int code, const DevReq &r, int role) {
  const int scheme = scheme_of(code), op = op_of(code), stage = stage_of(code);
  if (scheme <= 1) {
    if (r.gen && stage == 0 && op != OP_DEC) draw_coins(key, r, const_cast<uint8_t *>(r.in0));
    const fdev::Inst v = frodo_view(r);
    if (op == OP_KEYPAIR) {
      if (stage == 0) fdev::kp_prologue_inst(v);
      else fdev::pk_hash_inst(v);
    } else if (op == OP_ENC) {
      if (stage == 0) fdev::prologue_inst<OP_ENC>(v);
      else fdev::ss_inst<OP_ENC>(v);
    } else {
      if (stage == 1 && role == 0) fdev::prologue_inst<OP_DEC>(v);
      else if (stage == 1) fdev::ct_absorb_inst(v);
      else fdev::ss_inst<OP_DEC>(v);
    }
  } else if (scheme == 2) {
    saber_thread<2>(key, op, stage, r, role);
  } else if (scheme == 3) {
    saber_thread<3>(key, op, stage, r, role);
  } else {
    saber_thread<4>(key, op, stage, r, role);
  }
}

template <int L, int MODE>
__device__ __forceinline__ void saber_product(int form, const sdev::Inst &v, uint8_t *smem, uint32_t tbase,
                                              uint32_t *err) {
  if (form == FORM_TC) sdev::product_tc_cta<L, MODE>(v, smem, tbase, err);
  else if (form == FORM_INT32) sdev::product_dp4a_cta<L, MODE, true>(v, smem);
  else sdev::product_dp4a_cta<L, MODE, false>(v, smem);
}

template <int L>
__device__ __forceinline__ void saber_cta(int op, int stage, int tc, const DevReq &r, uint8_t *smem, uint32_t tbase,
                                          uint32_t *err) {
  const sdev::Inst v = saber_view<L>(r);
  if (op == OP_KEYPAIR) saber_product<L, sdev::PM_KEYPAIR>(tc, v, smem, tbase, err);
  else if (op == OP_ENC) saber_product<L, sdev::PM_ENC>(tc, v, smem, tbase, err);
  else if (stage == 0) saber_product<L, sdev::PM_DEC_INNER>(tc, v, smem, tbase, err);
  else saber_product<L, sdev::PM_DEC_CMP>(tc, v, smem, tbase, err);
}

constexpr int kTcStages = 2;

// Frodo CTA stages with row generator GT (tcgen05 stage, NST tile stages) / GD (others).
template <class GT, class GD, int NST>
__device__ __forceinline__ void frodo_cta(int op, int stage, int tc, const DevReq &r, uint8_t *smem, uint32_t tbase,
                                          uint32_t *err) {
  const fdev::Inst v = frodo_view(r);
  if (op == OP_KEYPAIR) {
    if (tc == FORM_TC) fdev::kp_as_tc_cta<NST == 2 ? fdev::KPT_NST : 1, GT>(v, smem, tbase, err);
    else if (tc == FORM_INT32) fdev::kp_as_dp4a_cta<true, GT>(v, smem);
    else fdev::kp_as_dp4a_cta<false, GT>(v, smem);
  } else if (op == OP_ENC) {
    if (tc == FORM_TC) fdev::sa_tc_cta<OP_ENC, NST, GT>(v, smem, tbase, err);
    else if (tc == FORM_INT32) fdev::sa_dp4a_cta<OP_ENC, true, GD>(v, smem);
    else fdev::sa_dp4a_cta<OP_ENC, false, GD>(v, smem);
  } else if (stage == 0) {
    fdev::dec_w_cta(v, smem);
  } else {
    if (tc == FORM_TC) fdev::sa_tc_cta<OP_DEC, NST, GT>(v, smem, tbase, err);
    else if (tc == FORM_INT32) fdev::sa_dp4a_cta<OP_DEC, true, GD>(v, smem);
    else fdev::sa_dp4a_cta<OP_DEC, false, GD>(v, smem);
  }
}

__device__ __forceinline__ void cta_stage(int code, const DevReq &r, uint8_t *smem, uint32_t tbase, uint32_t *err) {
  const int scheme = scheme_of(code), op = op_of(code), stage = stage_of(code);
  const int tc = form_of(code);  // product form (FORM_DP4A / FORM_INT32 / FORM_TC)
  if (scheme == 0) {
    frodo_cta<fdev::ShakeRows, fdev::ShakeRows, kTcStages>(op, stage, tc, r, smem, tbase, err);
  } else if (scheme == 1) {  // FrodoKEM-976-AES (one tile stage: see frodo.cu)
    frodo_cta<fdev::AesRowsFull, fdev::AesRowsHalf, 1>(op, stage, tc, r, smem, tbase, err);
  } else if (scheme == 2) {
    saber_cta<2>(op, stage, tc, r, smem, tbase, err);
  } else if (scheme == 3) {
    saber_cta<3>(op, stage, tc, r, smem, tbase, err);
  } else {
    saber_cta<4>(op, stage, tc, r, smem, tbase, err);
  }
}

constexpr int kSmem = std::max({fdev::TcLayout<kTcStages>::total, fdev::DP4A_SMEM, fdev::DEC_W_SMEM,
                                fdev::KP_AS_SMEM, fdev::KptLayout::total, sdev::PL<4>::TC_TOTAL, sdev::PL<3>::TC_TOTAL,
                                sdev::PL<2>::TC_TOTAL,
                                // FrodoKEM-976-AES stages: layout + AES table copies
                                fdev::TcLayout<1>::total + fdev::AesRowsFull::SMEM,
                                fdev::DP4A_SMEM + fdev::AesRowsHalf::SMEM, fdev::KP_AS_SMEM + fdev::AesRowsFull::SMEM,
                                fdev::KptLayoutT<1>::total + fdev::AesRowsFull::SMEM});
static_assert(kSmem == fdev::TcLayout<kTcStages>::total, "the AES stages must not raise the kernel's shared memory");


}  // namespace mixed
}  // namespace dpkem
