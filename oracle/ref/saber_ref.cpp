/*
 * Saber (level REF_SABER_L) keypair / encaps / decaps assembled from the reference's own
 * kernels (SABER-GPU/src/poly.cu, pack.cu), compiled as host C++ through cuda_emu.h and run
 * at one instance per call.
 *
 * TEST INFRASTRUCTURE ONLY: it generates golden vectors that pin the oracle's restatement
 * (oracle/saber.c) to the reference's code.  Encaps and decaps follow the reference's
 * launch sequence (SABER-GPU/src/cuda_kernel.cu:68-133 and :213-273) with its launch shapes
 * at one instance, on zeroed buffers (the products accumulate with +=).  Glue here replaces
 * only what cannot give the specification's result:
 *   - shake128_gpu (poly.cu:897-1010) is warp-synchronous shared-memory code (not emulable,
 *     and its tail input is not offset per instance); GenMatrix runs as the reference's
 *     serial GenMatrix_gpu / GenMatrix_gpu2 (poly.cu:1012-1039) instead;
 *   - verify_gpu / cmov_gpu (pack.cu:225-255) keep per-byte flags and never move (and the
 *     reference runs cmov after hashing, cuda_kernel.cu:272-273); the compare and the
 *     conditional move of z are done here in the specification's order (cmov, then hash);
 *   - the eT = 3 / 6 branches of POLT2BS_gpu / BS2POLT_gpu are commented out in the
 *     reference (pack.cu:105-132, :165-197); for LightSaber and FireSaber the eT-bit
 *     little-endian packing of c_m is done here (Saber l=3 uses the reference's packers);
 *   - the reference has no key generation (its keys come from tv.h); keypair here is built
 *     from the reference's pieces: seed_A = shake128(coins[0:32]) and GenMatrix, GenSecret,
 *     the product DoDP4Av7 on the transposed matrix, post_process and POLVECp2BS_gpu; only the
 *     13-bit packing of the secret into sk (which the reference only ever unpacks, with
 *     BS2POLVECq_gpu) is glue;
 *   - the encaps message is SHA3-256 of the coins (cuda_kernel.cu:68), the reference's
 *     d_m being tv.h's copy of that value.
 */
#include "cuda_emu.h"

#include "src/poly.cu"
#include "src/pack.cu"

namespace {

constexpr int L = SABER_L, N = SABER_N;
constexpr int PKB = SABER_INDCPA_PUBLICKEYBYTES, SKB = SABER_SECRETKEYBYTES, CTB = SABER_BYTES_CCA_DEC;
constexpr int PVC = SABER_POLYVECCOMPRESSEDBYTES;

// Little-endian bit packing of `bits`-bit values (glue, see the header).
void bitpack(uint8_t *out, const uint16_t *v, int count, int bits) {
  memset(out, 0, (size_t)count * bits / 8);
  for (int i = 0; i < count; ++i)
    for (int b = 0; b < bits; ++b)
      if ((v[i] >> b) & 1) out[(i * bits + b) / 8] |= (uint8_t)(1u << ((i * bits + b) % 8));
}

void bitunpack(uint16_t *v, const uint8_t *in, int count, int bits) {
  for (int i = 0; i < count; ++i) {
    v[i] = 0;
    for (int b = 0; b < bits; ++b) v[i] |= (uint16_t)(((in[(i * bits + b) / 8] >> ((i * bits + b) % 8)) & 1) << b);
  }
}

void pack_cm(uint8_t *out, uint16_t *vp) {  // c_m into the ciphertext tail
  if (SABER_ET == 4) {
    KLAUNCH(POLT2BS_gpu, 1, N / 2, out, vp);  // cuda_kernel.cu:129
  } else {
    uint16_t t[N];
    for (int i = 0; i < N; ++i) t[i] = vp[i] & ((1u << SABER_ET) - 1);
    bitpack(out, t, N, SABER_ET);
  }
}

void unpack_cm(uint16_t *cm, uint8_t *in) {
  if (SABER_ET == 4)
    KLAUNCH(BS2POLT_gpu, 1, N / 2, in, cm);  // cuda_kernel.cu:226
  else
    bitunpack(cm, in, N, SABER_ET);
}

// IND-CPA encryption of m (32 bytes) with noise seed `seed_sp` under pk, into ct:
// cuda_kernel.cu:73-129 (and its copy in decaps, :236-265).
void indcpa_enc(uint8_t *ct, uint8_t *m, uint8_t *seed_sp, uint8_t *pk) {
  std::vector<uint16_t> A(L * L * N), sp(L * N), bp(L * N, 0), b(L * N, 0), vp(N, 0), mp(N, 0);
  std::vector<short2> a1(L * L * N / 2), a2(L * L * N / 2);
  std::vector<char4> pb(L * N / 2);
  KLAUNCH(GenSecret_gpu, 1, 1, sp.data(), seed_sp);                                       // :73
  KLAUNCH(GenMatrix_gpu2, 1, 1, A.data(), pk + PVC);                                       // :75-76 (serial form)
  KLAUNCH(packdp2av2, 1, N / 2, a1.data(), a2.data(), A.data());                           // :82
  KLAUNCH(packdp2b, 1, N / 2, pb.data(), sp.data());                                       // :83
  KLAUNCH(DoDP4Av7, 1, N / 2, bp.data(), a1.data(), a2.data(), pb.data());                 // :84
  KLAUNCH(post_process, 1, N, bp.data());                                                  // :89
  KLAUNCH(POLVECp2BS_gpu, 1, N / 4, ct, bp.data());                                        // :91
  KLAUNCH(BS2POLVECp_gpu, 1, N / 4, pk, b.data(), (uint32_t)PKB);                         // :92
  KLAUNCH(packdp2av2Inner, 1, N / 2, a1.data(), a2.data(), b.data());                      // :109
  KLAUNCH(packdp2b, 1, N / 2, pb.data(), sp.data());                                       // :110
  KLAUNCH(DoDP4Av7_inner, 1, N / 2, vp.data(), a1.data(), a2.data(), pb.data());           // :111
  KLAUNCH(BS2POLmsg_gpu, 1, SABER_KEYBYTES, m, mp.data());                                 // :127
  KLAUNCH(post_process2, 1, N, vp.data(), mp.data());                                      // :128
  pack_cm(ct + PVC, vp.data());                                                            // :129
}

}  // namespace

#define REF_CAT2(a, b) a##b
#define REF_CAT(a, b) REF_CAT2(a, b)
#define REF_FN(name) REF_CAT(REF_CAT(ref_saber, SABER_L), _##name)

extern "C" {

// coins = seed_A source (32) || noise seed (32) || z (32)
int REF_FN(keypair)(uint8_t *pk, uint8_t *sk, const uint8_t *coins) {
  std::vector<uint8_t> c(coins, coins + 96), seed_a(SABER_SEEDBYTES);
  std::vector<uint16_t> A(L * L * N), At(L * L * N), s(L * N), b(L * N, 0);
  std::vector<short2> a1(L * L * N / 2), a2(L * L * N / 2);
  std::vector<char4> pb(L * N / 2);
  std::vector<uint8_t> d_pk(PKB, 0), d_sk(SKB, 0);
  KLAUNCH(shake128, 1, 1, seed_a.data(), (unsigned long long)SABER_SEEDBYTES, c.data(),
          (unsigned long long)SABER_SEEDBYTES);
  KLAUNCH(GenMatrix_gpu, 1, 1, A.data(), seed_a.data());
  KLAUNCH(GenSecret_gpu, 1, 1, s.data(), c.data() + 32);
  for (int i = 0; i < L; ++i)  // b = A^T s: the reference's product on the transposed matrix
    for (int j = 0; j < L; ++j) memcpy(&At[(i * L + j) * N], &A[(j * L + i) * N], 2 * N);
  KLAUNCH(packdp2av2, 1, N / 2, a1.data(), a2.data(), At.data());
  KLAUNCH(packdp2b, 1, N / 2, pb.data(), s.data());
  KLAUNCH(DoDP4Av7, 1, N / 2, b.data(), a1.data(), a2.data(), pb.data());
  KLAUNCH(post_process, 1, N, b.data());
  KLAUNCH(POLVECp2BS_gpu, 1, N / 4, d_pk.data(), b.data());
  memcpy(d_pk.data() + PVC, seed_a.data(), SABER_SEEDBYTES);
  std::vector<uint16_t> s13(L * N);
  for (int i = 0; i < L * N; ++i) s13[i] = s[i] & 0x1FFF;
  bitpack(d_sk.data(), s13.data(), L * N, SABER_EQ);
  std::vector<uint16_t> check(L * N, 0);
  KLAUNCH(BS2POLVECq_gpu, 1, N / 8, d_sk.data(), check.data());  // the reference's unpacker inverts it
  if (memcmp(check.data(), s13.data(), 2 * L * N)) return -1;
  memcpy(d_sk.data() + SABER_POLYVECBYTES, d_pk.data(), PKB);
  KLAUNCH(sha3_256_gpu, 1, 1, d_sk.data() + SKB - 64, d_pk.data(), (unsigned long long)PKB, (uint32_t)PKB, 64u);
  memcpy(d_sk.data() + SKB - 32, c.data() + 64, 32);
  memcpy(pk, d_pk.data(), PKB);
  memcpy(sk, d_sk.data(), SKB);
  return 0;
}

// coins = 32 bytes of encaps randomness (the reference's buf_tv[0:32])
int REF_FN(enc)(uint8_t *ct, uint8_t *ss, const uint8_t *pk, const uint8_t *coins) {
  std::vector<uint8_t> buf(64, 0), kr(64, 0), d_pk(pk, pk + PKB), d_c(CTB, 0), m(32);
  memcpy(buf.data(), coins, 32);
  KLAUNCH(sha3_256_gpu, 1, 1, buf.data(), buf.data(), 32ull, 64u, 64u);                    // :68
  KLAUNCH(sha3_256_gpu, 1, 1, buf.data() + 32, d_pk.data(), (unsigned long long)PKB, (uint32_t)PKB, 64u);  // :69
  KLAUNCH(sha3_512_gpu, 1, 1, kr.data(), buf.data(), 64ull);                               // :70
  memcpy(m.data(), buf.data(), 32);
  indcpa_enc(d_c.data(), m.data(), kr.data() + 32, d_pk.data());
  KLAUNCH(sha3_256_gpu, 1, 1, kr.data() + 32, d_c.data(), (unsigned long long)CTB, (uint32_t)CTB, 64u);   // :132
  KLAUNCH(sha3_256_gpu, 1, 1, ss, kr.data(), 64ull, 64u, 32u);                             // :133
  memcpy(ct, d_c.data(), CTB);
  return 0;
}

int REF_FN(dec)(uint8_t *ss, const uint8_t *ct, const uint8_t *sk) {
  std::vector<uint8_t> d_sk(sk, sk + SKB), d_c(ct, ct + CTB), m(32, 0), buf(64, 0), kr(64, 0), cmp(CTB, 0);
  std::vector<uint16_t> s(L * N, 0), b(L * N, 0), v(N, 0), cm(N, 0);
  std::vector<short2> a1(L * N / 2), a2(L * N / 2);
  std::vector<char4> pb(L * N / 2);
  KLAUNCH(BS2POLVECq_gpu, 1, N / 8, d_sk.data(), s.data());                                // :213
  KLAUNCH(BS2POLVECp_gpu, 1, N / 4, d_c.data(), b.data(), (uint32_t)CTB);                 // :214
  KLAUNCH(packdp2av2Inner, 1, N / 2, a1.data(), a2.data(), b.data());                      // :219
  KLAUNCH(packdp2b, 1, N / 2, pb.data(), s.data());                                        // :220
  KLAUNCH(DoDP4Av7_inner, 1, N / 2, v.data(), a1.data(), a2.data(), pb.data());            // :221
  unpack_cm(cm.data(), d_c.data() + PVC);                                                  // :226
  KLAUNCH(post_process3, 1, N, v.data(), cm.data());                                       // :227
  KLAUNCH(POLmsg2BS_gpu, 1, SABER_KEYBYTES, m.data(), v.data());                          // :228
  KLAUNCH(copysk, 1, 32, buf.data(), m.data(), d_sk.data());                               // :231
  KLAUNCH(sha3_512_gpu, 1, 1, kr.data(), buf.data(), 64ull);                               // :232
  std::vector<uint8_t> pk(d_sk.begin() + SABER_POLYVECBYTES, d_sk.begin() + SABER_POLYVECBYTES + PKB);
  indcpa_enc(cmp.data(), m.data(), kr.data() + 32, pk.data());                             // :236-265
  uint8_t diff = 0;  // :268 and :273 in the specification's form: compare, then move z before hashing
  for (int i = 0; i < CTB; ++i) diff |= d_c[i] ^ cmp[i];
  const uint8_t mask = (uint8_t)(0u - (uint32_t)(diff != 0));
  for (int i = 0; i < 32; ++i) kr[i] ^= mask & (kr[i] ^ d_sk[SKB - 32 + i]);
  KLAUNCH(sha3_256_gpu, 1, 1, kr.data() + 32, d_c.data(), (unsigned long long)CTB, (uint32_t)CTB, 64u);   // :270
  KLAUNCH(sha3_256_gpu, 1, 1, ss, kr.data(), 64ull, 64u, (uint32_t)SABER_KEYBYTES);       // :272
  return 0;
}

}  // extern "C"
