/*
 * CPU oracle: Keccak-f[1600] sponge, SHA3-256/512 and SHAKE128/256.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the parity checker and the timed CPU
 * baseline; no product code path links or calls it.
 *
 * Restated from FIPS 202 (round constants from the rc(t) LFSR, rotation offsets
 * from the (x,y) -> (y, 2x+3y) walk) rather than from tables.  It follows the
 * reference's sponge conventions: lanes are little-endian, absorb pads with the
 * domain byte p at the message tail and 0x80 in the last rate byte, squeeze emits
 * whole rate blocks (SABER-GPU/src/poly.cu:706-749, FrodoKEM976-GPU/src/shake.cu:337-377).
 * Pinned against Python hashlib in tests/test_oracle_hash.py.
 */
#include "oracle.h"

#include <string.h>

static uint64_t g_rc[24];
static int g_rot[25];
static int g_inited = 0;

static void keccak_tables(void) {
  if (g_inited) return;
  /* rc(t): LFSR over GF(2) with polynomial x^8 + x^6 + x^5 + x^4 + 1. */
  uint8_t r = 1;
  for (int ir = 0; ir < 24; ir++) {
    uint64_t c = 0;
    for (int j = 0; j < 7; j++) {
      if (r & 1) c |= 1ULL << ((1 << j) - 1);
      r = (r & 0x80) ? (uint8_t)((r << 1) ^ 0x71) : (uint8_t)(r << 1);
    }
    g_rc[ir] = c;
  }
  int x = 1, y = 0;
  g_rot[0] = 0;
  for (int t = 0; t < 24; t++) {
    g_rot[x + 5 * y] = ((t + 1) * (t + 2) / 2) % 64;
    int nx = y, ny = (2 * x + 3 * y) % 5;
    x = nx;
    y = ny;
  }
  g_inited = 1;
}

static inline uint64_t rotl64(uint64_t v, int n) { return n ? (v << n) | (v >> (64 - n)) : v; }

void oracle_keccak_f1600(uint64_t a[25]) {
  keccak_tables();
  uint64_t c[5], d[5], b[25];
  for (int ir = 0; ir < 24; ir++) {
    for (int xx = 0; xx < 5; xx++) c[xx] = a[xx] ^ a[xx + 5] ^ a[xx + 10] ^ a[xx + 15] ^ a[xx + 20];
    for (int xx = 0; xx < 5; xx++) d[xx] = c[(xx + 4) % 5] ^ rotl64(c[(xx + 1) % 5], 1);
    for (int i = 0; i < 25; i++) a[i] ^= d[i % 5];
    for (int xx = 0; xx < 5; xx++)
      for (int yy = 0; yy < 5; yy++)
        b[yy + 5 * ((2 * xx + 3 * yy) % 5)] = rotl64(a[xx + 5 * yy], g_rot[xx + 5 * yy]);
    for (int yy = 0; yy < 5; yy++)
      for (int xx = 0; xx < 5; xx++)
        a[xx + 5 * yy] = b[xx + 5 * yy] ^ (~b[(xx + 1) % 5 + 5 * yy] & b[(xx + 2) % 5 + 5 * yy]);
    a[0] ^= g_rc[ir];
  }
}

static inline uint64_t load_le64(const uint8_t *p) {
  uint64_t v = 0;
  for (int i = 7; i >= 0; i--) v = (v << 8) | p[i];
  return v;
}

static inline void store_le64(uint8_t *p, uint64_t v) {
  for (int i = 0; i < 8; i++) p[i] = (uint8_t)(v >> (8 * i));
}

void oracle_sponge_init(oracle_sponge *s, unsigned rate, uint8_t domain) {
  memset(s->a, 0, sizeof(s->a));
  s->rate = rate;
  s->domain = domain;
  s->pos = 0;
  s->squeezing = 0;
}

void oracle_sponge_absorb(oracle_sponge *s, const uint8_t *in, size_t len) {
  while (len > 0) {
    size_t take = s->rate - s->pos;
    if (take > len) take = len;
    for (size_t i = 0; i < take; i++) {
      size_t p = s->pos + i;
      s->a[p >> 3] ^= (uint64_t)in[i] << (8 * (p & 7));
    }
    s->pos += (unsigned)take;
    in += take;
    len -= take;
    if (s->pos == s->rate) {
      oracle_keccak_f1600(s->a);
      s->pos = 0;
    }
  }
}

static void sponge_finalize(oracle_sponge *s) {
  s->a[s->pos >> 3] ^= (uint64_t)s->domain << (8 * (s->pos & 7));
  s->a[(s->rate - 1) >> 3] ^= 0x80ULL << (8 * ((s->rate - 1) & 7));
  s->squeezing = 1;
  s->pos = s->rate; /* forces a permutation before the first output byte */
}

void oracle_sponge_squeeze(oracle_sponge *s, uint8_t *out, size_t len) {
  if (!s->squeezing) sponge_finalize(s);
  while (len > 0) {
    if (s->pos == s->rate) {
      oracle_keccak_f1600(s->a);
      s->pos = 0;
    }
    size_t take = s->rate - s->pos;
    if (take > len) take = len;
    for (size_t i = 0; i < take; i++) {
      size_t p = s->pos + i;
      out[i] = (uint8_t)(s->a[p >> 3] >> (8 * (p & 7)));
    }
    s->pos += (unsigned)take;
    out += take;
    len -= take;
  }
}

static void xof(unsigned rate, uint8_t dom, uint8_t *out, size_t outlen, const uint8_t *in, size_t inlen) {
  oracle_sponge s;
  oracle_sponge_init(&s, rate, dom);
  oracle_sponge_absorb(&s, in, inlen);
  oracle_sponge_squeeze(&s, out, outlen);
}

void oracle_shake128(uint8_t *out, size_t outlen, const uint8_t *in, size_t inlen) { xof(168, 0x1F, out, outlen, in, inlen); }
void oracle_shake256(uint8_t *out, size_t outlen, const uint8_t *in, size_t inlen) { xof(136, 0x1F, out, outlen, in, inlen); }
void oracle_sha3_256(uint8_t *out, const uint8_t *in, size_t inlen) { xof(136, 0x06, out, 32, in, inlen); }
void oracle_sha3_512(uint8_t *out, const uint8_t *in, size_t inlen) { xof(72, 0x06, out, 64, in, inlen); }

/* Seeded synthetic coins: SHAKE256(K || LE64(i) || tag, len), K = 00 01 .. 1F. */
void oracle_coins(uint8_t *out, size_t len, uint64_t index, const char *tag) {
  uint8_t buf[32 + 8 + 64];
  size_t n = 0;
  for (int i = 0; i < 32; i++) buf[n++] = (uint8_t)i;
  for (int i = 0; i < 8; i++) buf[n++] = (uint8_t)(index >> (8 * i));
  size_t tl = strlen(tag);
  if (tl > 64) tl = 64;
  memcpy(buf + n, tag, tl);
  n += tl;
  oracle_shake256(out, len, buf, n);
}

void oracle_coins_batch(uint8_t *out, size_t len, uint64_t first, size_t count, const char *tag) {
  for (size_t i = 0; i < count; i++) oracle_coins(out + i * len, len, first + i, tag);
}
