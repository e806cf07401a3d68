/*
 * CPU oracle: AES-128 encryption (FIPS 197), for the A matrix of FrodoKEM-976-AES.
 *
 * TEST INFRASTRUCTURE ONLY (parity checker; never linked by the product).  The
 * reference declares an AES interface but ships no implementation
 * (FrodoKEM976-GPU/include/aes.h, gen_a_mat_mul.cuh:6-7) and does not vendor PQClean's
 * aes.c, so this restates the standard: the S-box is the multiplicative inverse in
 * GF(2^8) (modulus x^8 + x^4 + x^3 + x + 1) followed by the affine map with constant
 * 0x63; the key schedule, SubBytes, ShiftRows, MixColumns and AddRoundKey follow the
 * standard's byte-level definitions.  Pinned against Python's `cryptography` AES-ECB
 * (tests/test_oracle_aes.py).
 */
#include <pthread.h>
#include <string.h>

#include "oracle.h"

static uint8_t g_sbox[256];
static pthread_once_t g_once = PTHREAD_ONCE_INIT;

static uint8_t xtime(uint8_t a) { return (uint8_t)((a << 1) ^ ((a & 0x80) ? 0x1B : 0x00)); }

static uint8_t gf_mul(uint8_t a, uint8_t b) {
  uint8_t r = 0;
  while (b) {
    if (b & 1) r ^= a;
    a = xtime(a);
    b >>= 1;
  }
  return r;
}

static uint8_t rotl8(uint8_t b, int k) { return (uint8_t)((b << k) | (b >> (8 - k))); }

static void init_sbox(void) {
  for (int x = 0; x < 256; x++) {
    uint8_t inv = 0; /* 0 maps to 0 */
    if (x) {         /* x^254 = x^-1 */
      uint8_t p = (uint8_t)x, r = 1;
      for (int e = 254; e; e >>= 1) {
        if (e & 1) r = gf_mul(r, p);
        p = gf_mul(p, p);
      }
      inv = r;
    }
    g_sbox[x] = (uint8_t)(inv ^ rotl8(inv, 1) ^ rotl8(inv, 2) ^ rotl8(inv, 3) ^ rotl8(inv, 4) ^ 0x63);
  }
}

void oracle_aes128_expand(uint8_t rk[176], const uint8_t key[16]) {
  pthread_once(&g_once, init_sbox);
  memcpy(rk, key, 16);
  uint8_t rcon = 1;
  for (int i = 4; i < 44; i++) {
    uint8_t t[4];
    memcpy(t, rk + 4 * (i - 1), 4);
    if (i % 4 == 0) { /* RotWord, SubWord, Rcon */
      const uint8_t t0 = t[0];
      t[0] = (uint8_t)(g_sbox[t[1]] ^ rcon);
      t[1] = g_sbox[t[2]];
      t[2] = g_sbox[t[3]];
      t[3] = g_sbox[t0];
      rcon = xtime(rcon);
    }
    for (int b = 0; b < 4; b++) rk[4 * i + b] = (uint8_t)(rk[4 * (i - 4) + b] ^ t[b]);
  }
}

void oracle_aes128_encrypt(uint8_t out[16], const uint8_t in[16], const uint8_t rk[176]) {
  uint8_t s[16]; /* s[r + 4c] = state[r][c] */
  for (int i = 0; i < 16; i++) s[i] = (uint8_t)(in[i] ^ rk[i]);
  for (int round = 1; round <= 10; round++) {
    uint8_t t[16];
    for (int c = 0; c < 4; c++) /* SubBytes and ShiftRows: row r moves left by r */
      for (int r = 0; r < 4; r++) t[r + 4 * c] = g_sbox[s[r + 4 * ((c + r) & 3)]];
    if (round < 10) {
      for (int c = 0; c < 4; c++) { /* MixColumns */
        const uint8_t a0 = t[4 * c], a1 = t[4 * c + 1], a2 = t[4 * c + 2], a3 = t[4 * c + 3];
        s[4 * c] = (uint8_t)(xtime(a0) ^ (xtime(a1) ^ a1) ^ a2 ^ a3);
        s[4 * c + 1] = (uint8_t)(a0 ^ xtime(a1) ^ (xtime(a2) ^ a2) ^ a3);
        s[4 * c + 2] = (uint8_t)(a0 ^ a1 ^ xtime(a2) ^ (xtime(a3) ^ a3));
        s[4 * c + 3] = (uint8_t)((xtime(a0) ^ a0) ^ a1 ^ a2 ^ xtime(a3));
      }
    } else {
      memcpy(s, t, 16);
    }
    for (int i = 0; i < 16; i++) s[i] ^= rk[16 * round + i];
  }
  memcpy(out, s, 16);
}

void oracle_aes128_ecb(uint8_t *out, const uint8_t *in, size_t blocks, const uint8_t key[16]) {
  uint8_t rk[176];
  oracle_aes128_expand(rk, key);
  for (size_t b = 0; b < blocks; b++) oracle_aes128_encrypt(out + 16 * b, in + 16 * b, rk);
}
