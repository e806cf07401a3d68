"""The five measured workloads at their full sizes, checked for bit-exactness:

1. FrodoKEM-976, 128 instances: keypair -> encaps -> decaps against the CPU oracle byte for
   byte, plus 128 tampered decaps (implicit rejection).
2. Saber l=3, 4096 instances: tcgen05 vs dp4a vs INT32 on every instance, the CPU oracle on
   a 512-instance stride sample.
3. FrodoKEM-976, 8192 instances: keypairs on the GPU spot-checked against the oracle on 256
   instances, encaps+decaps with every form compared on every instance.
4. 16384 mixed requests (4 schemes x 3 ops, shuffled) in one persistent launch, equal to
   the batched calls on every request.
(5, the serving loop, is covered by test_gpu_serving.py.)
"""
import os

import numpy as np
import pytest
import torch

import dpcrypto_b200 as d

pytestmark = pytest.mark.gpu
FORMS = [d.FORM_TC, d.FORM_DP4A, d.FORM_INT32]
THREADS = os.cpu_count() or 8


def _tamper(ct):
    bad = ct.copy()
    for i in range(bad.shape[0]):
        bad[i, (i * 7919) % bad.shape[1]] ^= 1 << (i % 8)
    return bad


def test_frodo_128_against_oracle(engine, oracle):
    n = 128
    kc, ec = oracle.coins(n, 64, "kp"), oracle.coins(n, 24, "enc")
    pk_o, sk_o = oracle.keypair(0, kc, threads=THREADS)
    ct_o, ss_o = oracle.enc(0, pk_o, ec, threads=THREADS)
    bad = _tamper(ct_o)
    rej_o = oracle.dec(0, bad, sk_o, threads=THREADS)
    for form in (d.FORM_DP4A, d.FORM_TC):
        pk, sk = engine.keypair(d.FRODO976, kc, form)
        assert (pk == pk_o).all() and (sk == sk_o).all()
        ct, ss = engine.enc(d.FRODO976, pk, ec, form)
        assert (ct == ct_o).all() and (ss == ss_o).all()
        assert (engine.dec(d.FRODO976, ct, sk, form) == ss_o).all()
        rej = engine.dec(d.FRODO976, bad, sk, form)
        assert (rej == rej_o).all()
        assert not (rej == ss_o).all(axis=1).any()


def test_saber_l3_4096_forms_and_sample(engine, oracle):
    n = 4096
    kc = torch.empty((n, 96), dtype=torch.uint8, device="cuda")
    ec = torch.empty((n, 32), dtype=torch.uint8, device="cuda")
    engine.coins(n, 96, "kp", out=kc)
    engine.coins(n, 32, "enc", out=ec)
    res = {}
    for form in FORMS:
        pk, sk = engine.keypair(d.SABER, kc, form)
        ct, ss = engine.enc(d.SABER, pk, ec, form)
        bad = ct.clone()
        bad[::2, 17] ^= 4
        ss_dec, ss_bad = engine.dec(d.SABER, ct, sk, form), engine.dec(d.SABER, bad, sk, form)
        torch.cuda.synchronize()
        res[form] = [t.cpu().numpy() for t in (pk, sk, ct, ss, ss_dec, bad, ss_bad)]
        assert (res[form][4] == res[form][3]).all()
    for form in FORMS[1:]:
        for a, b in zip(res[FORMS[0]], res[form]):
            assert (a == b).all()
    pk, sk, ct, ss, _, bad, ss_bad = res[FORMS[0]]
    idx = np.arange(0, n, n // 512)
    h_kc, h_ec = kc.cpu().numpy()[idx], ec.cpu().numpy()[idx]
    pk_o, sk_o = oracle.keypair(3, h_kc, threads=THREADS)
    assert (pk[idx] == pk_o).all() and (sk[idx] == sk_o).all()
    ct_o, ss_o = oracle.enc(3, pk_o, h_ec, threads=THREADS)
    assert (ct[idx] == ct_o).all() and (ss[idx] == ss_o).all()
    assert (ss_bad[idx] == oracle.dec(3, bad[idx], sk_o, threads=THREADS)).all()


def test_frodo_8192_spot_and_forms(engine, oracle):
    n = 8192
    kc = torch.empty((n, 64), dtype=torch.uint8, device="cuda")
    ec = torch.empty((n, 24), dtype=torch.uint8, device="cuda")
    engine.coins(n, 64, "kp", out=kc)
    engine.coins(n, 24, "enc", out=ec)
    pk, sk = engine.keypair(d.FRODO976, kc, d.FORM_TC)
    pk2, sk2 = engine.keypair(d.FRODO976, kc, d.FORM_DP4A)
    assert torch.equal(pk, pk2) and torch.equal(sk, sk2)
    del pk2, sk2
    ct, ss = engine.enc(d.FRODO976, pk, ec, d.FORM_TC)
    for form in FORMS[1:]:
        ct2, ss2 = engine.enc(d.FRODO976, pk, ec, form)
        assert torch.equal(ct, ct2) and torch.equal(ss, ss2)
    del ct2, ss2
    for form in FORMS:
        assert torch.equal(engine.dec(d.FRODO976, ct, sk, form), ss)
    idx = torch.arange(0, n, n // 256, device="cuda")
    h_kc, h_ec = kc[idx].cpu().numpy(), ec[idx].cpu().numpy()
    pk_o, sk_o = oracle.keypair(0, h_kc, threads=THREADS)
    assert (pk[idx].cpu().numpy() == pk_o).all() and (sk[idx].cpu().numpy() == sk_o).all()
    ct_o, ss_o = oracle.enc(0, pk_o, h_ec, threads=THREADS)
    assert (ct[idx].cpu().numpy() == ct_o).all() and (ss[idx].cpu().numpy() == ss_o).all()


@pytest.mark.parametrize("form", FORMS)
def test_mixed_16384(engine, form, oracle_check_items):
    from dpcrypto_b200.workloads import MixedBatch

    mb = MixedBatch(engine, 16384, seed=3)
    engine.mixed(mb.items, form)
    engine.sync()
    torch.cuda.synchronize()
    assert mb.check()
    # a stride sample (every scheme and op) recomputed by the oracle from the request inputs
    assert oracle_check_items(mb.items, stride=97, offset=FORMS.index(form)) >= 160
