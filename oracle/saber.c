/*
 * CPU oracle: Saber KEM (round 3) for LightSaber (l=2, mu=10, eT=3), Saber (l=3,
 * mu=8, eT=4) and FireSaber (l=4, mu=6, eT=6).
 *
 * TEST INFRASTRUCTURE ONLY (parity checker and CPU baseline; never linked by the
 * product).  Saber l=3 is pinned against SABER-GPU/include/tv.h (tests/golden);
 * l=2 and l=4 are parity-unpinned (the reference compiles only l=3 correctly:
 * its eT=3/6 packers are commented out, SABER-GPU/src/pack.cu:105-132,165-197).
 *
 * Follows the reference's data flow and byte conventions:
 *  - parameters and byte sizes: SABER-GPU/include/params.h:4-48
 *  - h1/h2 rounding constants and post-processing: SABER-GPU/src/poly.cu:11-12,360-382
 *  - GenMatrix = SHAKE128(seed_A, l*l*416) unpacked 13-bit LE: poly.cu:1012-1038, pack.cu:51-65
 *  - GenSecret = CBD_mu(SHAKE128(seed, l*mu*32)): poly.cu:815-895,1041-1052
 *  - encaps flow (m = SHA3-256(coins), kr = SHA3-512(m||H(pk)), enc with kr[32:],
 *    k = SHA3-256(kr[0:32]||SHA3-256(c))): SABER-GPU/src/cuda_kernel.cu:19-153
 *  - decaps flow: cuda_kernel.cu:155-299, in the specification order (cmov of z
 *    before the final hash; the reference hashes first, cuda_kernel.cu:272-273)
 *  - LSB-first bit packing at 13/10/eT/1 bits: pack.cu:8-212
 *  - keygen uses the transposed product (b = A^T s), encaps the plain one.
 */
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define SN 256
#define EQ 13
#define EP 10

typedef struct {
  int l, mu, et;
} saber_params;

static int params_for(int level, saber_params *p) {
  switch (level) {
    case 2: p->l = 2; p->mu = 10; p->et = 3; return 0;
    case 3: p->l = 3; p->mu = 8; p->et = 4; return 0;
    case 4: p->l = 4; p->mu = 6; p->et = 6; return 0;
    default: return -1;
  }
}

static size_t polyvec_bytes(const saber_params *p) { return (size_t)p->l * EQ * SN / 8; }
static size_t polyveccomp_bytes(const saber_params *p) { return (size_t)p->l * EP * SN / 8; }
static size_t pk_bytes(const saber_params *p) { return polyveccomp_bytes(p) + 32; }
static size_t sk_bytes(const saber_params *p) { return polyvec_bytes(p) + pk_bytes(p) + 64; }
static size_t ct_bytes(const saber_params *p) { return polyveccomp_bytes(p) + (size_t)p->et * SN / 8; }

int oracle_saber_sizes(int level, size_t *pk, size_t *sk, size_t *ct, size_t *ss) {
  saber_params p;
  if (params_for(level, &p)) return -1;
  if (pk) *pk = pk_bytes(&p);
  if (sk) *sk = sk_bytes(&p);
  if (ct) *ct = ct_bytes(&p);
  if (ss) *ss = 32;
  return 0;
}

/* LSB-first bit packing of n values, `bits` bits each. */
static void bitpack(uint8_t *out, const uint16_t *in, size_t n, int bits) {
  size_t nbytes = (n * bits + 7) / 8;
  memset(out, 0, nbytes);
  size_t pos = 0;
  for (size_t i = 0; i < n; i++) {
    uint32_t v = in[i] & ((1u << bits) - 1);
    for (int b = 0; b < bits; b++, pos++) out[pos >> 3] |= (uint8_t)(((v >> b) & 1) << (pos & 7));
  }
}

static void bitunpack(uint16_t *out, const uint8_t *in, size_t n, int bits) {
  size_t pos = 0;
  for (size_t i = 0; i < n; i++) {
    uint32_t v = 0;
    for (int b = 0; b < bits; b++, pos++) v |= (uint32_t)((in[pos >> 3] >> (pos & 7)) & 1) << b;
    out[i] = (uint16_t)v;
  }
}

/* res += a * b in Z_{2^16}[x]/(x^256 + 1). */
void oracle_saber_polmul_acc(const uint16_t *a, const uint16_t *b, uint16_t *res) {
  uint32_t acc[SN];
  for (int i = 0; i < SN; i++) acc[i] = res[i];
  /* x^i * x^j = x^(i+j), and x^(i+j) = -x^(i+j-256) once i + j wraps: two branch-free
   * loops per a[i], the second subtracting. */
  for (int i = 0; i < SN; i++) {
    const uint32_t ai = a[i];
    for (int j = 0; j < SN - i; j++) acc[i + j] += ai * b[j];
    for (int j = SN - i; j < SN; j++) acc[i + j - SN] -= ai * b[j];
  }
  for (int i = 0; i < SN; i++) res[i] = (uint16_t)acc[i];
}

void oracle_saber_genmatrix(int level, uint16_t *a, const uint8_t *seed) {
  saber_params p;
  if (params_for(level, &p)) return;
  size_t polyb = EQ * SN / 8, len = (size_t)p.l * p.l * polyb;
  uint8_t *buf = (uint8_t *)malloc(len);
  oracle_shake128(buf, len, seed, 32);
  for (int k = 0; k < p.l * p.l; k++) bitunpack(a + (size_t)k * SN, buf + k * polyb, SN, EQ);
  free(buf);
}

/* Centered binomial sample: coefficient c = popcount(first mu/2 bits) - popcount(next mu/2). */
static void cbd(uint16_t *s, const uint8_t *buf, int mu) {
  int half = mu / 2;
  size_t pos = 0;
  for (int c = 0; c < SN; c++) {
    int a = 0, b = 0;
    for (int t = 0; t < half; t++, pos++) a += (buf[pos >> 3] >> (pos & 7)) & 1;
    for (int t = 0; t < half; t++, pos++) b += (buf[pos >> 3] >> (pos & 7)) & 1;
    s[c] = (uint16_t)(a - b);
  }
}

void oracle_saber_gensecret(int level, uint16_t *s, const uint8_t *seed) {
  saber_params p;
  if (params_for(level, &p)) return;
  size_t coinb = (size_t)p.mu * SN / 8, len = (size_t)p.l * coinb;
  uint8_t *buf = (uint8_t *)malloc(len);
  oracle_shake128(buf, len, seed, 32);
  for (int i = 0; i < p.l; i++) cbd(s + (size_t)i * SN, buf + i * coinb, p.mu);
  free(buf);
}

void oracle_saber_matvec(int level, uint16_t *res, const uint16_t *a, const uint16_t *s, int transpose) {
  saber_params p;
  if (params_for(level, &p)) return;
  memset(res, 0, sizeof(uint16_t) * p.l * SN);
  for (int i = 0; i < p.l; i++)
    for (int j = 0; j < p.l; j++) {
      const uint16_t *aij = a + ((size_t)(transpose ? j * p.l + i : i * p.l + j)) * SN;
      oracle_saber_polmul_acc(aij, s + (size_t)j * SN, res + (size_t)i * SN);
    }
}

static void indcpa_enc(const saber_params *p, int level, uint8_t *ct, const uint8_t *m, const uint8_t *seed_sp,
                       const uint8_t *pk) {
  int l = p->l;
  const uint16_t h1 = 1 << (EQ - EP - 1);
  uint16_t *a = (uint16_t *)malloc(sizeof(uint16_t) * l * l * SN);
  uint16_t *sp = (uint16_t *)malloc(sizeof(uint16_t) * l * SN);
  uint16_t *bp = (uint16_t *)malloc(sizeof(uint16_t) * l * SN);
  uint16_t *b = (uint16_t *)malloc(sizeof(uint16_t) * l * SN);
  uint16_t vp[SN];
  oracle_saber_genmatrix(level, a, pk + polyveccomp_bytes(p));
  oracle_saber_gensecret(level, sp, seed_sp);
  oracle_saber_matvec(level, bp, a, sp, 0);
  for (int i = 0; i < l * SN; i++) bp[i] = (uint16_t)((bp[i] + h1) >> (EQ - EP));
  bitpack(ct, bp, (size_t)l * SN, EP);
  bitunpack(b, pk, (size_t)l * SN, EP);
  memset(vp, 0, sizeof vp);
  for (int j = 0; j < l; j++) oracle_saber_polmul_acc(b + j * SN, sp + j * SN, vp);
  for (int i = 0; i < SN; i++) {
    uint16_t mbit = (m[i >> 3] >> (i & 7)) & 1;
    vp[i] = (uint16_t)((uint16_t)(vp[i] - (mbit << (EP - 1)) + h1) >> (EP - p->et));
  }
  bitpack(ct + polyveccomp_bytes(p), vp, SN, p->et);
  free(a);
  free(sp);
  free(bp);
  free(b);
}

int oracle_saber_keypair(int level, uint8_t *pk, uint8_t *sk, const uint8_t *coins) {
  saber_params p;
  if (params_for(level, &p)) return -1;
  int l = p.l;
  const uint16_t h1 = 1 << (EQ - EP - 1);
  uint8_t seed_a[32];
  uint16_t *a = (uint16_t *)malloc(sizeof(uint16_t) * l * l * SN);
  uint16_t *s = (uint16_t *)malloc(sizeof(uint16_t) * l * SN);
  uint16_t *b = (uint16_t *)malloc(sizeof(uint16_t) * l * SN);
  oracle_shake128(seed_a, 32, coins, 32);
  oracle_saber_genmatrix(level, a, seed_a);
  oracle_saber_gensecret(level, s, coins + 32);
  oracle_saber_matvec(level, b, a, s, 1);
  for (int i = 0; i < l * SN; i++) b[i] = (uint16_t)((b[i] + h1) >> (EQ - EP));
  bitpack(sk, s, (size_t)l * SN, EQ);
  bitpack(pk, b, (size_t)l * SN, EP);
  memcpy(pk + polyveccomp_bytes(&p), seed_a, 32);
  size_t pkb = pk_bytes(&p), skb = sk_bytes(&p);
  memcpy(sk + polyvec_bytes(&p), pk, pkb);
  oracle_sha3_256(sk + skb - 64, pk, pkb);
  memcpy(sk + skb - 32, coins + 64, 32);
  free(a);
  free(s);
  free(b);
  return 0;
}

int oracle_saber_enc(int level, uint8_t *ct, uint8_t *ss, const uint8_t *pk, const uint8_t *coins) {
  saber_params p;
  if (params_for(level, &p)) return -1;
  uint8_t buf[64], kr[64];
  oracle_sha3_256(buf, coins, 32);
  oracle_sha3_256(buf + 32, pk, pk_bytes(&p));
  oracle_sha3_512(kr, buf, 64);
  indcpa_enc(&p, level, ct, buf, kr + 32, pk);
  oracle_sha3_256(kr + 32, ct, ct_bytes(&p));
  oracle_sha3_256(ss, kr, 64);
  return 0;
}

int oracle_saber_dec(int level, uint8_t *ss, const uint8_t *ct, const uint8_t *sk) {
  saber_params p;
  if (params_for(level, &p)) return -1;
  int l = p.l;
  const uint16_t h2 = (1 << (EP - 2)) - (1 << (EP - p.et - 1)) + (1 << (EQ - EP - 1));
  size_t ctb = ct_bytes(&p), skb = sk_bytes(&p);
  uint16_t *s = (uint16_t *)malloc(sizeof(uint16_t) * l * SN);
  uint16_t *b = (uint16_t *)malloc(sizeof(uint16_t) * l * SN);
  uint16_t v[SN], cm[SN];
  uint8_t buf[64], kr[64];
  uint8_t *cmp = (uint8_t *)malloc(ctb);
  bitunpack(s, sk, (size_t)l * SN, EQ);
  bitunpack(b, ct, (size_t)l * SN, EP);
  memset(v, 0, sizeof v);
  for (int j = 0; j < l; j++) oracle_saber_polmul_acc(b + j * SN, s + j * SN, v);
  bitunpack(cm, ct + polyveccomp_bytes(&p), SN, p.et);
  memset(buf, 0, 32);
  for (int i = 0; i < SN; i++) {
    uint16_t t = (uint16_t)((uint16_t)(v[i] + h2 - (cm[i] << (EP - p.et))) >> (EP - 1));
    buf[i >> 3] |= (uint8_t)((t & 1) << (i & 7));
  }
  memcpy(buf + 32, sk + skb - 64, 32);
  oracle_sha3_512(kr, buf, 64);
  indcpa_enc(&p, level, cmp, buf, kr + 32, sk + polyvec_bytes(&p));
  uint8_t diff = 0;
  for (size_t i = 0; i < ctb; i++) diff |= ct[i] ^ cmp[i];
  uint8_t mask = (uint8_t)(0 - (uint8_t)(((uint32_t)diff + 0xFFu) >> 8)); /* 0xFF iff diff != 0 */
  oracle_sha3_256(kr + 32, ct, ctb);
  for (int i = 0; i < 32; i++) kr[i] = (uint8_t)((kr[i] & ~mask) | (sk[skb - 32 + i] & mask));
  oracle_sha3_256(ss, kr, 64);
  free(s);
  free(b);
  free(cmp);
  return 0;
}
