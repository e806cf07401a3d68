"""FrodoKEM-976-SHAKE on the GPU through the C ABI, byte for byte against the CPU oracle."""
import hashlib

import numpy as np
import pytest

import dpcrypto_b200 as d

pytestmark = pytest.mark.gpu
FORMS = [d.FORM_DP4A, d.FORM_INT32, d.FORM_TC]


def _tamper(ct):
    bad = ct.copy()
    for i in range(bad.shape[0]):
        bad[i, (i * 7919) % bad.shape[1]] ^= 1 << (i % 8)
    return bad


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("n", [1, 3])
def test_frodo_matches_oracle(engine, oracle, form, n):
    kc, ec = oracle.coins(n, 64, "kp", first=11), oracle.coins(n, 24, "enc", first=11)
    pk_o, sk_o = oracle.keypair(0, kc, threads=8)
    ct_o, ss_o = oracle.enc(0, pk_o, ec, threads=8)
    pk, sk = engine.keypair(d.FRODO976, kc, form)
    assert (pk == pk_o).all() and (sk == sk_o).all()
    ct, ss = engine.enc(d.FRODO976, pk_o, ec, form)
    assert (ct == ct_o).all()
    assert (ss == ss_o).all()
    assert (engine.dec(d.FRODO976, ct_o, sk_o, form) == ss_o).all()
    bad = _tamper(ct_o)
    assert (engine.dec(d.FRODO976, bad, sk_o, form) == oracle.dec(0, bad, sk_o, threads=8)).all()


def test_frodo_forms_agree_at_scale(engine, oracle):
    n = 300
    kc, ec = oracle.coins(n, 64, "kp", first=1000), oracle.coins(n, 24, "enc", first=1000)
    pk, sk = engine.keypair(d.FRODO976, kc, d.FORM_DP4A)
    pk2, sk2 = engine.keypair(d.FRODO976, kc, d.FORM_TC)
    assert (pk == pk2).all() and (sk == sk2).all()
    ct, ss = engine.enc(d.FRODO976, pk, ec, d.FORM_TC)
    ct2, ss2 = engine.enc(d.FRODO976, pk, ec, d.FORM_DP4A)
    assert (ct == ct2).all() and (ss == ss2).all()
    for form in FORMS:
        assert (engine.dec(d.FRODO976, ct, sk, form) == ss).all()
        bad = _tamper(ct)
        rej = engine.dec(d.FRODO976, bad, sk, form)
        for i in (0, 1, n - 1):
            assert rej[i].tobytes() == hashlib.shake_256(bad[i].tobytes() + sk[i, :24].tobytes()).digest(24)
    # spot-check instances spread over the batch against the oracle
    idx = np.array([0, 137, n - 1])
    pk_o, _ = oracle.keypair(0, kc[idx], threads=3)
    assert (pk[idx] == pk_o).all()
    ct_o, ss_o = oracle.enc(0, pk[idx], ec[idx], threads=3)
    assert (ct[idx] == ct_o).all() and (ss[idx] == ss_o).all()


@pytest.mark.parametrize("form", [d.FORM_TC, d.FORM_DP4A])
@pytest.mark.parametrize("layout", ["one", "five", "warp"])
def test_frodo_sponges_on_several_lanes(engine, oracle, form, layout):
    """Every thread-level sponge stage (keypair prologue, H(pk), both prologues, the
    ciphertext pre-absorb and both final hashes) on one lane, five lanes per state or a warp
    per state, against the oracle; n = 7 leaves a partial group of lanes, and tampered
    ciphertexts take the reject path."""
    from dpcrypto_b200 import kem

    big = 1 << 30
    sel = {"one": dict(frodo_warp_max=0, frodo_ss_warp_max=0, frodo_five_max=0, frodo_ss_five_max=0),
           "five": dict(frodo_warp_max=0, frodo_ss_warp_max=0, frodo_five_max=big, frodo_ss_five_max=big),
           "warp": dict(frodo_warp_max=big, frodo_ss_warp_max=big)}[layout]
    with kem.knobs(**sel):
        n = 7
        kc, ec = oracle.coins(n, 64, "kp", first=61), oracle.coins(n, 24, "enc", first=61)
        pk_o, sk_o = oracle.keypair(0, kc, threads=8)
        ct_o, ss_o = oracle.enc(0, pk_o, ec, threads=8)
        pk, sk = engine.keypair(d.FRODO976, kc, form)
        assert (pk == pk_o).all() and (sk == sk_o).all()
        ct, ss = engine.enc(d.FRODO976, pk_o, ec, form)
        assert (ct == ct_o).all() and (ss == ss_o).all()
        assert (engine.dec(d.FRODO976, ct_o, sk_o, form) == ss_o).all()
        bad = _tamper(ct_o)
        assert (engine.dec(d.FRODO976, bad, sk_o, form) == oracle.dec(0, bad, sk_o, threads=8)).all()
