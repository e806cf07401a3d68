/*
 * CPU oracle for the batched FrodoKEM-976-SHAKE / Saber KEM path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for parity tests, __graft_entry__.smoke()
 * and the CPU-baseline leg of bench.py.  No product code path may link or call it.
 *
 * The reference (DPCrypto) has no CPU implementation and does not vendor the
 * PQClean sources its headers name, so this is a restatement of the published
 * FrodoKEM (round 3, SHAKE and AES variants) and Saber (round 3) algorithms, following the
 * reference's data flow and byte layouts (file:line citations in each .c file).
 * Saber l=3 is pinned by SABER-GPU/include/tv.h; Keccak by Python hashlib;
 * FrodoKEM-976 and LightSaber/FireSaber have no fixture in the reference
 * (parity for those rests on round trips and on CPU == GPU agreement).
 */
#ifndef DPKEM_ORACLE_H
#define DPKEM_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Keccak / SHA-3 ---- */
typedef struct {
  uint64_t a[25];
  unsigned rate, pos;
  uint8_t domain;
  int squeezing;
} oracle_sponge;

void oracle_keccak_f1600(uint64_t a[25]);        /* unrolled, used by the sponge */
void oracle_keccak_f1600_plain(uint64_t a[25]);  /* loop form, the cross-check */
void oracle_sponge_init(oracle_sponge *s, unsigned rate, uint8_t domain);
void oracle_sponge_absorb(oracle_sponge *s, const uint8_t *in, size_t len);
void oracle_sponge_squeeze(oracle_sponge *s, uint8_t *out, size_t len);
void oracle_shake128(uint8_t *out, size_t outlen, const uint8_t *in, size_t inlen);
void oracle_shake256(uint8_t *out, size_t outlen, const uint8_t *in, size_t inlen);
void oracle_sha3_256(uint8_t *out, const uint8_t *in, size_t inlen);
void oracle_sha3_512(uint8_t *out, const uint8_t *in, size_t inlen);
void oracle_coins(uint8_t *out, size_t len, uint64_t index, const char *tag);
void oracle_coins_batch(uint8_t *out, size_t len, uint64_t first, size_t count, const char *tag);

/* ---- FrodoKEM-976-SHAKE ---- */
#define ORACLE_FRODO_PK 15632
#define ORACLE_FRODO_SK 31296
#define ORACLE_FRODO_CT 15744
#define ORACLE_FRODO_SS 24
#define ORACLE_FRODO_KP_COINS 64
#define ORACLE_FRODO_ENC_COINS 24

int oracle_frodo_keypair(uint8_t *pk, uint8_t *sk, const uint8_t *coins);
int oracle_frodo_enc(uint8_t *ct, uint8_t *ss, const uint8_t *pk, const uint8_t *coins);
int oracle_frodo_dec(uint8_t *ss, const uint8_t *ct, const uint8_t *sk);
/* Row i of A as 976 uint16 values (SHAKE128 / AES-128 variant). */
void oracle_frodo_gen_row(uint16_t *row, const uint8_t *seed_a, int i);
void oracle_frodo_gen_row_aes(uint16_t *row, const uint8_t *seed_a, int i);
/* aes = 0: FrodoKEM-976-SHAKE, 1: FrodoKEM-976-AES (same sizes and layouts). */
int oracle_frodo_keypair_v(uint8_t *pk, uint8_t *sk, const uint8_t *coins, int aes);
int oracle_frodo_enc_v(uint8_t *ct, uint8_t *ss, const uint8_t *pk, const uint8_t *coins, int aes);
int oracle_frodo_dec_v(uint8_t *ss, const uint8_t *ct, const uint8_t *sk, int aes);

/* ---- AES-128 (FIPS 197) ---- */
void oracle_aes128_expand(uint8_t rk[176], const uint8_t key[16]);
void oracle_aes128_encrypt(uint8_t out[16], const uint8_t in[16], const uint8_t rk[176]);
void oracle_aes128_ecb(uint8_t *out, const uint8_t *in, size_t blocks, const uint8_t key[16]);
void oracle_frodo_sample(uint16_t *s, size_t n);

/* ---- Saber (level = 2 LightSaber, 3 Saber, 4 FireSaber) ---- */
int oracle_saber_sizes(int level, size_t *pk, size_t *sk, size_t *ct, size_t *ss);
int oracle_saber_keypair(int level, uint8_t *pk, uint8_t *sk, const uint8_t *coins);
int oracle_saber_enc(int level, uint8_t *ct, uint8_t *ss, const uint8_t *pk, const uint8_t *coins);
int oracle_saber_dec(int level, uint8_t *ss, const uint8_t *ct, const uint8_t *sk);
/* Internals exposed for pinning against the reference fixture. */
void oracle_saber_genmatrix(int level, uint16_t *a, const uint8_t *seed);
void oracle_saber_gensecret(int level, uint16_t *s, const uint8_t *seed);
void oracle_saber_matvec(int level, uint16_t *res, const uint16_t *a, const uint16_t *s, int transpose);
void oracle_saber_polmul_acc(const uint16_t *a, const uint16_t *b, uint16_t *res);

/* ---- Threaded batch drivers (CPU baseline) ----
 * op: 0 keypair, 1 enc, 2 dec.  scheme: 0 Frodo-976, 2/3/4 Saber level.
 * in0/in1/out0/out1 follow the single-instance argument order of the op. */
int oracle_batch(int scheme, int op, size_t n, int nthreads, uint8_t *out0, uint8_t *out1,
                 const uint8_t *in0, const uint8_t *in1);

#ifdef __cplusplus
}
#endif
#endif
