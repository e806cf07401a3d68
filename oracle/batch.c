/*
 * CPU oracle: threaded batch driver, used only as the timed CPU baseline
 * (bench.py cpu_baseline and --impl reference) and by tests.  One KEM instance
 * per work item, instances split into contiguous ranges over pthreads.  The
 * reference has no CPU path (its hosts only orchestrate GPU launches,
 * FrodoKEM976-GPU/src/cuda_kernel.cu, SABER-GPU/src/cuda_kernel.cu), so this
 * restatement stands in for "the reference's CPU implementation of the path".
 */
#include <pthread.h>
#include <stdlib.h>

#include "oracle.h"

typedef struct {
  int scheme, op;
  size_t begin, end;
  uint8_t *out0, *out1;
  const uint8_t *in0, *in1;
  size_t s_out0, s_out1, s_in0, s_in1;
  int status;
} work_t;

static int sizes(int scheme, int op, size_t *o0, size_t *o1, size_t *i0, size_t *i1) {
  size_t pk, sk, ct, ss;
  if (scheme == 0 || scheme == 1) {
    pk = ORACLE_FRODO_PK; sk = ORACLE_FRODO_SK; ct = ORACLE_FRODO_CT; ss = ORACLE_FRODO_SS;
  } else if (oracle_saber_sizes(scheme, &pk, &sk, &ct, &ss)) {
    return -1;
  }
  size_t kpc = scheme <= 1 ? ORACLE_FRODO_KP_COINS : 96, encc = scheme <= 1 ? ORACLE_FRODO_ENC_COINS : 32;
  switch (op) {
    case 0: *o0 = pk; *o1 = sk; *i0 = kpc; *i1 = 0; return 0;
    case 1: *o0 = ct; *o1 = ss; *i0 = pk; *i1 = encc; return 0;
    case 2: *o0 = ss; *o1 = 0; *i0 = ct; *i1 = sk; return 0;
    default: return -1;
  }
}

static void *run(void *arg) {
  work_t *w = (work_t *)arg;
  for (size_t i = w->begin; i < w->end; i++) {
    uint8_t *o0 = w->out0 + i * w->s_out0, *o1 = w->out1 ? w->out1 + i * w->s_out1 : NULL;
    const uint8_t *a = w->in0 + i * w->s_in0, *b = w->in1 ? w->in1 + i * w->s_in1 : NULL;
    int rc;
    if (w->scheme <= 1) { /* 0 FrodoKEM-976-SHAKE, 1 FrodoKEM-976-AES */
      const int aes = w->scheme;
      rc = w->op == 0   ? oracle_frodo_keypair_v(o0, o1, a, aes)
           : w->op == 1 ? oracle_frodo_enc_v(o0, o1, a, b, aes)
                        : oracle_frodo_dec_v(o0, a, b, aes);
    } else {
      rc = w->op == 0 ? oracle_saber_keypair(w->scheme, o0, o1, a)
           : w->op == 1 ? oracle_saber_enc(w->scheme, o0, o1, a, b)
                        : oracle_saber_dec(w->scheme, o0, a, b);
    }
    if (rc) w->status = rc;
  }
  return NULL;
}

int oracle_batch(int scheme, int op, size_t n, int nthreads, uint8_t *out0, uint8_t *out1, const uint8_t *in0,
                 const uint8_t *in1) {
  size_t so0, so1, si0, si1;
  if (sizes(scheme, op, &so0, &so1, &si0, &si1)) return -1;
  if (nthreads < 1) nthreads = 1;
  if ((size_t)nthreads > n) nthreads = n ? (int)n : 1;
  work_t *w = (work_t *)calloc((size_t)nthreads, sizeof(work_t));
  pthread_t *th = (pthread_t *)calloc((size_t)nthreads, sizeof(pthread_t));
  for (int t = 0; t < nthreads; t++) {
    w[t] = (work_t){scheme, op, n * t / nthreads, n * (t + 1) / nthreads, out0, out1, in0, in1,
                    so0, so1, si0, si1, 0};
    pthread_create(&th[t], NULL, run, &w[t]);
  }
  int status = 0;
  for (int t = 0; t < nthreads; t++) {
    pthread_join(th[t], NULL);
    if (w[t].status) status = w[t].status;
  }
  free(w);
  free(th);
  return status;
}
