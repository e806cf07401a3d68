"""FrodoKEM-976-AES on the GPU through the C ABI: byte for byte against the oracle (whose
AES-128 is pinned to the cryptography package), in every product form."""
import hashlib

import numpy as np
import pytest

import dpcrypto_b200 as d

pytestmark = pytest.mark.gpu
FORMS = [d.FORM_DP4A, d.FORM_INT32, d.FORM_TC]
AES = d.FRODO976AES


def _tamper(ct):
    bad = ct.copy()
    for i in range(bad.shape[0]):
        bad[i, (i * 7919) % bad.shape[1]] ^= 1 << (i % 8)
    return bad


@pytest.fixture(scope="module")
def aes_case(oracle):
    n = 2
    kc, ec = oracle.coins(n, 64, "kp", first=21), oracle.coins(n, 24, "enc", first=21)
    pk, sk = oracle.keypair(oracle.FRODO_AES, kc, threads=n)
    ct, ss = oracle.enc(oracle.FRODO_AES, pk, ec, threads=n)
    bad = _tamper(ct)
    rej = oracle.dec(oracle.FRODO_AES, bad, sk, threads=n)
    return kc, ec, pk, sk, ct, ss, bad, rej


@pytest.mark.parametrize("form", FORMS)
def test_frodo_aes_matches_oracle(engine, aes_case, form):
    kc, ec, pk_o, sk_o, ct_o, ss_o, bad, rej_o = aes_case
    pk, sk = engine.keypair(AES, kc, form)
    assert (pk == pk_o).all() and (sk == sk_o).all()
    ct, ss = engine.enc(AES, pk_o, ec, form)
    assert (ct == ct_o).all() and (ss == ss_o).all()
    assert (engine.dec(AES, ct_o, sk_o, form) == ss_o).all()
    assert (engine.dec(AES, bad, sk_o, form) == rej_o).all()


def test_frodo_aes_differs_from_shake(engine, aes_case):
    kc = aes_case[0]
    pk_a, _ = engine.keypair(AES, kc, d.FORM_TC)
    pk_s, _ = engine.keypair(d.FRODO976, kc, d.FORM_TC)
    assert (pk_a[:, :16] == pk_s[:, :16]).all()  # same seedA
    assert not (pk_a[:, 16:] == pk_s[:, 16:]).all(axis=1).any()  # other matrix A


def test_frodo_aes_forms_agree_at_scale(engine, oracle):
    n = 300
    kc, ec = oracle.coins(n, 64, "kp", first=400), oracle.coins(n, 24, "enc", first=400)
    pk, sk = engine.keypair(AES, kc, d.FORM_TC)
    for form in (d.FORM_DP4A, d.FORM_INT32):
        pk2, sk2 = engine.keypair(AES, kc, form)
        assert (pk == pk2).all() and (sk == sk2).all()
    ct, ss = engine.enc(AES, pk, ec, d.FORM_TC)
    for form in FORMS:
        ct2, ss2 = engine.enc(AES, pk, ec, form)
        assert (ct == ct2).all() and (ss == ss2).all()
        assert (engine.dec(AES, ct, sk, form) == ss).all()
        bad = _tamper(ct)
        rej = engine.dec(AES, bad, sk, form)
        for i in (0, n - 1):
            assert rej[i].tobytes() == hashlib.shake_256(bad[i].tobytes() + sk[i, :24].tobytes()).digest(24)
    idx = np.array([0, n - 1])
    pk_o, _ = oracle.keypair(oracle.FRODO_AES, kc[idx], threads=2)
    assert (pk[idx] == pk_o).all()
