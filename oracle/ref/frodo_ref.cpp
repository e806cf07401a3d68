/*
 * FrodoKEM-976-SHAKE keypair / encaps / decaps assembled from the reference's own kernels
 * (FrodoKEM976-GPU/src/*.cu), compiled as host C++ through cuda_emu.h and run at one
 * instance per call.
 *
 * TEST INFRASTRUCTURE ONLY: it generates golden vectors that pin the oracle's restatement
 * (oracle/frodo.c) to the reference's code.  Every arithmetic step below is a reference
 * kernel or device function, launched with the reference's launch shapes
 * (FrodoKEM976-GPU/src/cuda_kernel.cu:21-335), on buffers zeroed first.  The glue here
 * replaces only the steps whose reference form cannot give the specification's result:
 *   - shake256_gpu (shake.cu:495-604) is warp-synchronous shared-memory code without
 *     barriers (not emulable here, and it has the input-offset defect); SHAKE256 is run
 *     instead with the reference's serial sponge functions keccak_absorb_ser /
 *     keccak_squeezeblocks_ser (shake.cu:337-377) and its KeccakF1600_StatePermute;
 *   - shake128_ser (shake.cu:619-644) writes only the low byte of the row index and leaves
 *     the high byte uninitialised; rows of A here absorb LE16(i) || seedA through the same
 *     serial sponge functions;
 *   - ct_verify_gpu (util.cu:193-207) maps an OR of differences with bit 15 set to "equal"
 *     (its sign trick drops the shift of the constant-time compare), so decaps would accept
 *     tampered ciphertexts; the selector is computed here as the specification defines it and
 *     handed to the reference's ct_select_gpu;
 *   - the reference fills its coins with constants; here they are
 *     inputs, laid out s || seedSE || z (keypair) and mu (encaps) as the reference uses them
 *     (cuda_kernel.cu:51-53, :149-150).
 */
#include "cuda_emu.h"

#include "src/shake.cu"
#include "src/sample_pack.cu"
#include "src/encode_decode.cu"
#include "src/matrix_kernel.cu"
#include "src/util.cu"

namespace {

constexpr int N = PARAMS_N, NB = PARAMS_NBAR;
constexpr int PK = CRYPTO_PUBLICKEYBYTES, SK = CRYPTO_SECRETKEYBYTES, CT = CRYPTO_CIPHERTEXTBYTES;
constexpr int SS = CRYPTO_BYTES;

// SHAKE256(in, inlen) -> out[outlen] with the reference's serial sponge (rate 136, pad 0x1F).
void shake256_ref(uint8_t *out, size_t outlen, const uint8_t *in, size_t inlen) {
  uint64_t s[25] = {0};
  keccak_absorb_ser(s, 136, in, inlen, 0x1F);
  const size_t nblocks = outlen / 136;
  keccak_squeezeblocks_ser(out, nblocks, s, 136);
  if (outlen % 136) {
    uint8_t t[136];
    keccak_squeezeblocks_ser(t, 1, s, 136);
    memcpy(out + nblocks * 136, t, outlen % 136);
  }
}

// Row i of A (976 int16) = SHAKE128(LE16(i) || seedA), 1952 bytes, with the reference's serial
// sponge: the body of shake128_ser with both bytes of the row index set.
void gen_a_row(int16_t *row, const uint8_t *seed_a, int i) {
  uint8_t in[BYTES_SEED_A + 2];
  in[0] = (uint8_t)i;
  in[1] = (uint8_t)(i >> 8);
  memcpy(in + 2, seed_a, BYTES_SEED_A);
  uint64_t s[25] = {0};
  keccak_absorb_ser(s, SHAKE128_RATE, in, sizeof in, 0x1F);
  uint8_t out[12 * SHAKE128_RATE];
  keccak_squeezeblocks_ser(out, 12, s, SHAKE128_RATE);
  memcpy(row, out, 2 * N);
}

void gen_a(int16_t *A, const uint8_t *seed_a) {  // 976 x 976, row-major
  for (int i = 0; i < N; ++i) gen_a_row(A + (size_t)i * N, seed_a, i);
}

// The specification's constant-time compare (0 if equal, -1 otherwise).
int8_t selector(const uint16_t *a, const uint16_t *b, size_t len) {
  uint16_t r = 0;
  for (size_t i = 0; i < len; ++i) r |= a[i] ^ b[i];
  return (int8_t)((-(int32_t)r) >> 31);
}

struct Buffers {
  std::vector<int16_t> A = std::vector<int16_t>((size_t)N * N);
  std::vector<uint16_t> r = std::vector<uint16_t>((2 * N + NB) * NB);
};

}  // namespace

extern "C" {

// coins = s(24) || seedSE(24) || z(16)
int ref_frodo_keypair(uint8_t *pk, uint8_t *sk, const uint8_t *coins) {
  Buffers b;
  std::vector<uint8_t> randomness(coins, coins + 2 * SS + BYTES_SEED_A);
  std::vector<uint8_t> seed_se(1 + SS);
  std::vector<uint16_t> d_s(2 * N * NB, 0), B(N * NB, 0), S(N * NB, 0);
  std::vector<uint8_t> pkh(BYTES_PKHASH), d_pk(PK, 0), d_sk(SK, 0);
  seed_se[0] = 0x5F;
  memcpy(seed_se.data() + 1, randomness.data() + SS, SS);
  shake256_ref(d_pk.data(), BYTES_SEED_A, randomness.data() + 2 * SS, BYTES_SEED_A);     // :64
  shake256_ref((uint8_t *)d_s.data(), 2 * N * NB * 2, seed_se.data(), 1 + SS);           // :65
  KLAUNCH(copy_matrix_gpu_x2, 1, N, B.data(), d_s.data() + N * NB);                        // :67
  KLAUNCH(copy_matrix_gpu, 1, N, S.data(), d_s.data());                                    // :68
  KLAUNCH(sample_n_gpu, 1, N, S.data());                                                   // :69
  KLAUNCH(sample_n_gpu, 1, N, B.data());                                                   // :70
  gen_a(b.A.data(), d_pk.data());                                                          // :73-74
  KLAUNCH(as_plus_e_gpu, 1, N, B.data(), b.A.data(), S.data());                           // :77
  KLAUNCH(pack_gpu, 1, 488, d_pk.data(), (size_t)32, B.data(), (size_t)16, (uint8_t)PARAMS_LOGQ,
          (uint32_t)BYTES_SEED_A);                                                         // :79
  shake256_ref(pkh.data(), BYTES_PKHASH, d_pk.data(), PK);                                 // :80
  KLAUNCH(copy_sk_s, 1, SS, d_sk.data(), randomness.data());                               // :81
  KLAUNCH(copy_sk_pk, 1, 1024, d_sk.data(), d_pk.data());                                  // :82
  KLAUNCH(copy_sk_S, 1, 1024, d_sk.data(), (uint8_t *)S.data());                           // :83
  KLAUNCH(copy_sk_pkh, 1, 24, d_sk.data(), pkh.data());                                    // :84
  memcpy(pk, d_pk.data(), PK);
  memcpy(sk, d_sk.data(), SK);
  return 0;
}

// coins = mu (24 bytes)
int ref_frodo_enc(uint8_t *ct, uint8_t *ss, const uint8_t *pk, const uint8_t *coins) {
  Buffers b;
  std::vector<uint8_t> d_pk(pk, pk + PK), G2in(BYTES_PKHASH + BYTES_MU, 0), G2out(2 * SS), seed_se(1 + SS);
  std::vector<uint8_t> d_ct(CT, 0), Fin(CT + SS, 0);
  std::vector<uint16_t> Sp(N * NB, 0), Bp(N * NB, 0), Epp(NB * NB, 0), B(N * NB, 0), V(NB * NB, 0), C(NB * NB, 0);
  std::vector<char4> packed_sp(N * NB / 2);
  memcpy(G2in.data() + BYTES_PKHASH, coins, BYTES_MU);
  shake256_ref(G2in.data(), BYTES_PKHASH, d_pk.data(), PK);                                    // :159
  shake256_ref(G2out.data(), 2 * SS, G2in.data(), BYTES_PKHASH + BYTES_MU);                    // :160
  KLAUNCH(copy_seedSE, 1, SS, seed_se.data(), G2out.data());                                   // :161
  shake256_ref((uint8_t *)b.r.data(), b.r.size() * 2, seed_se.data(), 1 + SS);                 // :162
  KLAUNCH(copy_matrix_gpu_encap, 1, N, Bp.data(), b.r.data() + N * NB);                        // :164
  KLAUNCH(copy_matrix_gpu_encap_small, 1, 64, Epp.data(), b.r.data() + 2 * N * NB);            // :165
  KLAUNCH(copy_matrix_gpu_encap, 1, N, Sp.data(), b.r.data());                                 // :166
  KLAUNCH(sample_n_gpu, 1, N, Sp.data());                                                      // :167
  KLAUNCH(sample_n_gpu, 1, N, Bp.data());                                                      // :168
  KLAUNCH(sample_n_gpu_small, 1, NB * NB, Epp.data());                                         // :169
  gen_a(b.A.data(), d_pk.data());                                                              // :172-173
  KLAUNCH(packdp2bv2, 1, N / 2, packed_sp.data(), Sp.data());                                  // :175
  KLAUNCH(DoDP4Av5s, 1, N, (int16_t *)Bp.data(), (short2 *)b.A.data(), packed_sp.data());     // :176
  KLAUNCH(pack_gpu_encap, 1, 488, d_ct.data(), (size_t)32, Bp.data(), (size_t)16, (uint8_t)PARAMS_LOGQ,
          (uint32_t)0);                                                                        // :181
  KLAUNCH(unpack_gpu_encap, 1, 488, B.data(), (size_t)16, d_pk.data(), (size_t)32, (uint8_t)PARAMS_LOGQ,
          (uint32_t)BYTES_SEED_A);                                                             // :182
  KLAUNCH(mul_add_sb_plus_e_gpu, 1, NB, V.data(), B.data(), Sp.data(), Epp.data());            // :183
  KLAUNCH(key_encode_gpu, 1, NB, C.data(), (uint16_t *)G2in.data());                           // :184
  KLAUNCH(add_gpu, 1, NB * NB, C.data(), V.data(), C.data());                                  // :185
  KLAUNCH(pack_gpu_encap, 1, 4, d_ct.data() + (PARAMS_LOGQ * N * NB) / 8, (size_t)32, C.data(), (size_t)16,
          (uint8_t)PARAMS_LOGQ, (uint32_t)0);                                                  // :186
  KLAUNCH(copy_ct_encap, 1, N, Fin.data(), d_ct.data(), 0u, 0u, (uint32_t)CT, (uint32_t)(CT + SS),
          (uint32_t)CT);                                                                       // :187
  KLAUNCH(copy_ct_encap, 1, N, Fin.data(), G2out.data(), (uint32_t)SS, (uint32_t)CT, (uint32_t)(2 * SS),
          (uint32_t)(CT + SS), (uint32_t)SS);                                                  // :188
  shake256_ref(ss, SS, Fin.data(), CT + SS);                                                   // :189
  memcpy(ct, d_ct.data(), CT);
  return 0;
}

int ref_frodo_dec(uint8_t *ss, const uint8_t *ct, const uint8_t *sk) {
  Buffers b;
  std::vector<uint8_t> d_sk(sk, sk + SK), d_ct(ct, ct + CT), G2in(BYTES_PKHASH + BYTES_MU, 0), G2out(2 * SS);
  std::vector<uint8_t> seed_se(1 + SS), Fin(CT + SS, 0);
  std::vector<uint16_t> S(N * NB, 0), Bp(N * NB, 0), C(NB * NB, 0), W(NB * NB, 0), BBp(N * NB, 0), Sp(N * NB, 0);
  std::vector<uint16_t> Epp(NB * NB, 0), B(N * NB, 0), CC(NB * NB, 0);
  std::vector<char4> packed_sp(N * NB / 2);
  KLAUNCH(copy_u8_2_u16, 1, N, S.data(), d_sk.data(), 0u, (uint32_t)(SS + PK), (uint32_t)(N * NB), (uint32_t)SK,
          (uint32_t)(N * NB));                                                                 // :282
  KLAUNCH(unpack_gpu_decap, 1, 488, Bp.data(), (size_t)16, d_ct.data(), (size_t)32, (uint8_t)PARAMS_LOGQ, 0u,
          (uint32_t)(N * NB), (uint32_t)CT);                                                   // :284
  KLAUNCH(unpack_gpu_decap, 1, 4, C.data(), (size_t)16, d_ct.data(), (size_t)32, (uint8_t)PARAMS_LOGQ,
          (uint32_t)((PARAMS_LOGQ * N * NB) / 8), (uint32_t)(NB * NB), (uint32_t)CT);          // :285
  KLAUNCH(mul_bs_gpu, 1, NB, W.data(), Bp.data(), S.data());                                   // :286
  KLAUNCH(sub_gpu, 1, NB * NB, W.data(), C.data(), W.data());                                  // :287
  KLAUNCH(key_decode_gpu, 1, NB, (uint16_t *)G2in.data() + BYTES_PKHASH / 2, W.data());        // :288
  KLAUNCH(copy_vector, 1, BYTES_PKHASH, G2in.data(), d_sk.data(), 0u,
          (uint32_t)(SS + PK + 2 * N * NB), (uint32_t)(BYTES_PKHASH + BYTES_MU), (uint32_t)SK,
          (uint32_t)BYTES_PKHASH);                                                             // :289
  shake256_ref(G2out.data(), 2 * SS, G2in.data(), BYTES_PKHASH + BYTES_MU);                    // :290
  KLAUNCH(copy_seedSE, 1, SS, seed_se.data(), G2out.data());                                   // :291
  shake256_ref((uint8_t *)b.r.data(), b.r.size() * 2, seed_se.data(), 1 + SS);                 // :292
  KLAUNCH(copy_matrix_gpu_encap, 1, N, BBp.data(), b.r.data() + N * NB);                       // :293
  KLAUNCH(copy_matrix_gpu_encap, 1, N, Sp.data(), b.r.data());                                 // :294
  KLAUNCH(copy_matrix_gpu_encap_small, 1, 64, Epp.data(), b.r.data() + 2 * N * NB);            // :295
  KLAUNCH(sample_n_gpu, 1, N, Sp.data());                                                      // :296
  KLAUNCH(sample_n_gpu, 1, N, BBp.data());                                                     // :297
  KLAUNCH(sample_n_gpu_small, 1, NB * NB, Epp.data());                                         // :298
  gen_a(b.A.data(), d_sk.data() + 24);                                                         // :302-303
  KLAUNCH(packdp2bv2, 1, N / 2, packed_sp.data(), Sp.data());                                  // :306
  KLAUNCH(DoDP4Av5s, 1, N, (int16_t *)BBp.data(), (short2 *)b.A.data(), packed_sp.data());    // :307
  KLAUNCH(unpack_gpu_decap, 1, 488, B.data(), (size_t)16, d_sk.data(), (size_t)32, (uint8_t)PARAMS_LOGQ,
          (uint32_t)(SS + BYTES_SEED_A), (uint32_t)(N * NB), (uint32_t)SK);                   // :311
  KLAUNCH(mul_add_sb_plus_e_gpu, 1, NB, W.data(), B.data(), Sp.data(), Epp.data());            // :312
  KLAUNCH(key_encode_gpu, 1, NB, CC.data(), (uint16_t *)G2in.data());                          // :313
  KLAUNCH(add_gpu, 1, NB * NB, CC.data(), W.data(), CC.data());                                // :314
  KLAUNCH(copy_vector, 1, 1024, Fin.data(), d_ct.data(), 0u, 0u, (uint32_t)(CT + SS), (uint32_t)CT,
          (uint32_t)CT);                                                                       // :316
  KLAUNCH(reduce_q_gpu, 1, N, BBp.data());                                                     // :318
  // :319-321 with the specification's compare (ct_verify_gpu's defect, see the header)
  int8_t sel = (int8_t)(selector(Bp.data(), BBp.data(), N * NB) | selector(C.data(), CC.data(), NB * NB));
  KLAUNCH(ct_select_gpu, 1, SS, Fin.data() + CT, G2out.data() + SS, d_sk.data(), &sel);       // :322
  shake256_ref(ss, SS, Fin.data(), CT + SS);                                                   // :323
  return 0;
}

// Reference pieces on their own, for finer-grained checks of the restatement.
void ref_frodo_gen_a_row(uint16_t *row, const uint8_t *seed_a, int i) {
  gen_a_row(reinterpret_cast<int16_t *>(row), seed_a, i);
}

void ref_frodo_sample(uint16_t *s) {  // N * NB words in place
  KLAUNCH(sample_n_gpu, 1, N, s);
}

void ref_frodo_shake256(uint8_t *out, size_t outlen, const uint8_t *in, size_t inlen) {
  shake256_ref(out, outlen, in, inlen);
}

}  // extern "C"

extern "C" {
// The reference's ct_verify_gpu as it stands (util.cu:193-207): 0 = "equal", -1 = "differ".
// Kept callable so a test can record its defect (an OR of differences with bit 15 set is
// reported as equal).
int ref_frodo_ct_verify_raw(const uint16_t *a, const uint16_t *b, size_t len) {
  int8_t sel = 0;
  KLAUNCH(ct_verify_gpu, 1, 1, &sel, a, b, len);
  return sel;
}
}
