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
    """GenMatrix on one lane per state and on a lane pair (the saber_pair_max knob, with the
    five-lane and warp-per-state thresholds off) give the oracle's bytes, a partial last warp
    included."""
    from dpcrypto_b200 import kem

    with kem.knobs(saber_pair_max=pair_max, saber_warp_max=0, saber_five_max=0, saber_finish_warp_max=0,
                   saber_finish_five_max=0):
        n = 45
        kc, ec = oracle.coins(n, 96, "kp", first=77), oracle.coins(n, 32, "enc", first=77)
        pk_o, sk_o = oracle.keypair(level, kc, threads=8)
        ct_o, ss_o = oracle.enc(level, pk_o, ec, threads=8)
        pk, sk = engine.keypair(level, kc, d.FORM_TC)
        assert (pk == pk_o).all() and (sk == sk_o).all()
        ct, ss = engine.enc(level, pk_o, ec, d.FORM_TC)
        assert (ct == ct_o).all() and (ss == ss_o).all()
        assert (engine.dec(level, ct_o, sk_o, d.FORM_TC) == ss_o).all()


def _unpack13(b):
    bits = np.unpackbits(b, bitorder="little").reshape(-1, 13)
    return (bits.astype(np.int64) << np.arange(13)).sum(axis=1)


def _pack(v, width):
    bits = ((np.asarray(v, np.int64)[:, None] >> np.arange(width)) & 1).astype(np.uint8)
    return np.packbits(bits.ravel(), bitorder="little")


def _keypair_with_secret(oracle, level, seed_a, s, z):
    """A Saber key pair for a given secret vector s (centred integers), built from the
    oracle's GenMatrix and matrix-vector product: b = ((A^T s + h1) >> 3) mod 2^10,
    pk = pack10(b) || seed_A, sk = pack13(s) || pk || SHA3-256(pk) || z."""
    a = oracle.saber_genmatrix(level, seed_a)
    b = oracle.saber_matvec(level, a, (np.asarray(s) % 65536).astype(np.uint16), True)
    b = ((b.astype(np.int64) + 4) >> 3) & 0x3FF
    pk = np.concatenate([_pack(b, 10), np.frombuffer(seed_a, np.uint8)])
    sk = np.concatenate([_pack(np.asarray(s) % 8192, 13), pk, np.frombuffer(oracle.sha3_256(pk.tobytes()), np.uint8),
                         np.frombuffer(z, np.uint8)])
    return pk, sk


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("level", LEVELS)
def test_saber_malformed_secret_key(engine, oracle, level, form):
    """Secret keys whose secret coefficients lie outside the CBD range [-mu/2, mu/2] (a
    malformed sk; key generation never makes one).  Every form reads a secret coefficient as
    the low byte of its 13-bit field, sign-extended (the reference's DP path reads int8
    secrets the same way, SABER-GPU/src/poly.cu:56-68).  Recorded here:
    - coefficients inside [-128, 127]: the oracle's bytes, and decapsulation succeeds when the
      key pair was built for that secret (the secret is read exactly);
    - larger coefficients: the oracle's bytes for the key whose coefficients are replaced by
      their low byte."""
    n = 12
    kc, ec = oracle.coins(n, 96, "kp", first=31), oracle.coins(n, 32, "enc", first=31)
    rng = np.random.default_rng(level)
    mu_half = {2: 5, 3: 4, 4: 3}[level]
    nsec = 416 * level  # packed secret bytes at the start of sk
    pks, sks, wide, wide_lo = [], [], [], []
    for i in range(n):
        s = oracle.saber_gensecret(level, kc[i, 32:64].tobytes()).astype(np.int64)
        s = ((s + 4096) % 8192) - 4096  # centred
        pos = rng.choice(s.size, size=1 + i % 6, replace=False)
        # a few coefficients just outside the CBD range (small enough that decryption succeeds)
        s[pos] = rng.integers(mu_half + 1, mu_half + 12, size=pos.size) * rng.choice([-1, 1], size=pos.size)
        seed_a = oracle.shake128(kc[i, :32].tobytes(), 32)  # seed_A as key generation derives it
        pk, sk = _keypair_with_secret(oracle, level, seed_a, s, kc[i, 64:96].tobytes())
        pks.append(pk)
        sks.append(sk)
        w = s.copy()
        big = rng.integers(128, 4096, size=pos.size) * rng.choice([-1, 1], size=pos.size)
        w[pos] = big
        wk = sk.copy()
        wk[:nsec] = _pack(w % 8192, 13)
        wide.append(wk)
        w[pos] = ((big + 128) % 256) - 128  # the sign-extended low byte
        lk = sk.copy()
        lk[:nsec] = _pack(w % 8192, 13)
        wide_lo.append(lk)
    pk, sk, wide, wide_lo = (np.stack(x) for x in (pks, sks, wide, wide_lo))
    ct, ss = oracle.enc(level, pk, ec, threads=8)
    assert (oracle.dec(level, ct, sk, threads=8) == ss).all()  # the malformed key pairs work
    assert (engine.dec(level, ct, sk, form) == ss).all()
    ct_g, ss_g = engine.enc(level, pk, ec, form)
    assert (ct_g == ct).all() and (ss_g == ss).all()
    assert (engine.dec(level, ct, wide, form) == oracle.dec(level, ct, wide_lo, threads=8)).all()


@pytest.mark.parametrize("level", LEVELS)
@pytest.mark.parametrize("layout", ["one/pair", "five", "warp"])
def test_saber_sponges_on_several_lanes(engine, oracle, level, layout):
    """The prologue and finish sponges on one lane or a pair, five lanes per state
    (saber_five_max / saber_finish_five_max) or a warp per state (saber_warp_max /
    saber_finish_warp_max), against the oracle, with batch sizes that leave partial groups and
    partial warps (n = 1, 7, 45)."""
    from dpcrypto_b200 import kem

    big = 1 << 30
    sel = {"one/pair": dict(saber_warp_max=0, saber_finish_warp_max=0, saber_five_max=0, saber_finish_five_max=0),
           "five": dict(saber_warp_max=0, saber_finish_warp_max=0, saber_five_max=big, saber_finish_five_max=big),
           "warp": dict(saber_warp_max=big, saber_finish_warp_max=big)}[layout]
    with kem.knobs(**sel):
        for n in (1, 7, 45):
            kc, ec = oracle.coins(n, 96, "kp", first=91), oracle.coins(n, 32, "enc", first=91)
            pk_o, sk_o = oracle.keypair(level, kc, threads=8)
            ct_o, ss_o = oracle.enc(level, pk_o, ec, threads=8)
            for form in (d.FORM_TC, d.FORM_DP4A):
                pk, sk = engine.keypair(level, kc, form)
                assert (pk == pk_o).all() and (sk == sk_o).all()
                ct, ss = engine.enc(level, pk_o, ec, form)
                assert (ct == ct_o).all() and (ss == ss_o).all()
                assert (engine.dec(level, ct_o, sk_o, form) == ss_o).all()
                bad = _tamper(ct_o)
                assert (engine.dec(level, bad, sk_o, form) == oracle.dec(level, bad, sk_o, threads=8)).all()


@pytest.mark.parametrize("level", LEVELS)
@pytest.mark.parametrize("per_sm", [0, 1, 4, 5])
def test_saber_tc_product_persistent(engine, oracle, level, per_sm):
    """The tensor-core product with a CTA per instance (0) or as persistent CTAs that each
    take several instances and prefetch the next one's operands (1: 148 CTAs, so n = 333
    gives every CTA two or three instances), against the oracle, reject path included."""
    from dpcrypto_b200 import kem

    with kem.knobs(saber_tc_ctas_per_sm=per_sm):
        n = 333
        kc, ec = oracle.coins(n, 96, "kp", first=123), oracle.coins(n, 32, "enc", first=123)
        pk_o, sk_o = oracle.keypair(level, kc, threads=8)
        ct_o, ss_o = oracle.enc(level, pk_o, ec, threads=8)
        pk, sk = engine.keypair(level, kc, d.FORM_TC)
        assert (pk == pk_o).all() and (sk == sk_o).all()
        ct, ss = engine.enc(level, pk_o, ec, d.FORM_TC)
        assert (ct == ct_o).all() and (ss == ss_o).all()
        assert (engine.dec(level, ct_o, sk_o, d.FORM_TC) == ss_o).all()
        bad = _tamper(ct_o)
        assert (engine.dec(level, bad, sk_o, d.FORM_TC) == oracle.dec(level, bad, sk_o, threads=8)).all()
