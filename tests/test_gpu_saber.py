"""Saber (l = 2, 3, 4) on the GPU through the C ABI, byte for byte against the CPU oracle
and the reference fixture SABER-GPU/include/tv.h."""
import numpy as np
import pytest

import dpcrypto_b200 as d

pytestmark = pytest.mark.gpu
FORMS = [d.FORM_DP4A, d.FORM_INT32, d.FORM_TC]
LEVELS = [2, 3, 4]


def _tamper(ct):
    bad = ct.copy()
    for i in range(bad.shape[0]):
        bad[i, (i * 7919) % bad.shape[1]] ^= 1 << (i % 8)
    return bad


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("level", LEVELS)
@pytest.mark.parametrize("n", [1, 33, 200])
def test_saber_matches_oracle(engine, oracle, level, form, n):
    kc, ec = oracle.coins(n, 96, "kp", first=5), oracle.coins(n, 32, "enc", first=5)
    pk_o, sk_o = oracle.keypair(level, kc, threads=8)
    ct_o, ss_o = oracle.enc(level, pk_o, ec, threads=8)
    pk, sk = engine.keypair(level, kc, form)
    assert (pk == pk_o).all()
    assert (sk == sk_o).all()
    ct, ss = engine.enc(level, pk_o, ec, form)
    assert (ct == ct_o).all()
    assert (ss == ss_o).all()
    assert (engine.dec(level, ct_o, sk_o, form) == ss_o).all()
    bad = _tamper(ct_o)
    assert (engine.dec(level, bad, sk_o, form) == oracle.dec(level, bad, sk_o, threads=8)).all()


@pytest.mark.parametrize("form", FORMS)
def test_saber_reference_fixture(engine, oracle, saber_tv, form):
    pk, sk, buf = saber_tv["pk"][None].copy(), saber_tv["sk"][None].copy(), saber_tv["buf"][None, :32].copy()
    ct, ss = engine.enc(d.SABER, pk, buf, form)
    ct_o, ss_o = oracle.enc(3, pk, buf)
    assert (ct == ct_o).all() and (ss == ss_o).all()
    assert (engine.dec(d.SABER, ct, sk, form) == ss).all()


@pytest.mark.parametrize("level", LEVELS)
@pytest.mark.parametrize("pair_max", [0, 1 << 30])
def test_saber_prologue_lanes_per_state(engine, oracle, level, pair_max):
    """GenMatrix on one lane per state and on a lane pair (the saber_pair_max knob) give the
    oracle's bytes, a partial last warp included."""
    from dpcrypto_b200 import kem

    before = kem.get_tuning().get("saber_pair_max", 6144)
    kem.set_tuning("saber_pair_max", pair_max)
    try:
        n = 45
        kc, ec = oracle.coins(n, 96, "kp", first=77), oracle.coins(n, 32, "enc", first=77)
        pk_o, sk_o = oracle.keypair(level, kc, threads=8)
        ct_o, ss_o = oracle.enc(level, pk_o, ec, threads=8)
        pk, sk = engine.keypair(level, kc, d.FORM_TC)
        assert (pk == pk_o).all() and (sk == sk_o).all()
        ct, ss = engine.enc(level, pk_o, ec, d.FORM_TC)
        assert (ct == ct_o).all() and (ss == ss_o).all()
        assert (engine.dec(level, ct_o, sk_o, d.FORM_TC) == ss_o).all()
    finally:
        kem.set_tuning("saber_pair_max", before)
