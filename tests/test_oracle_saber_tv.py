"""Pin the Saber oracle to the reference's only known-answer fixture, SABER-GPU/include/tv.h
(copied into tests/golden/saber_l3_tv.npz by tests/golden/make_saber_tv.py)."""
import hashlib

import numpy as np


def _unpack(b, bits, count):
    v = np.unpackbits(np.asarray(b, np.uint8), bitorder="little")[: bits * count].reshape(count, bits)
    return (v.astype(np.uint32) << np.arange(bits, dtype=np.uint32)).sum(1)


def test_sk_layout(saber_tv):
    pk, sk = saber_tv["pk"], saber_tv["sk"]
    assert (sk[1248:2240] == pk).all()
    assert sk[2240:2272].tobytes() == hashlib.sha3_256(pk.tobytes()).digest()


def test_genmatrix(oracle, saber_tv):
    a = oracle.saber_genmatrix(3, saber_tv["pk"][960:992].tobytes())
    assert (a == saber_tv["A"]).all()


def test_message_and_secret(oracle, saber_tv):
    pk, buf = saber_tv["pk"], saber_tv["buf"]
    m = oracle.sha3_256(buf[:32].tobytes())
    assert m == saber_tv["m"].tobytes()
    kr = oracle.sha3_512(m + hashlib.sha3_256(pk.tobytes()).digest())
    assert (oracle.saber_gensecret(3, kr[32:64]) == saber_tv["sp"]).all()


def test_keygen_product(oracle, saber_tv):
    s = _unpack(saber_tv["sk"][:1248], 13, 768).astype(np.uint16)
    b = oracle.saber_matvec(3, saber_tv["A"], s, True).astype(np.uint32)
    assert (_unpack(saber_tv["pk"][:960], 10, 768) == ((b + 4) >> 3) & 0x3FF).all()


def test_fixture_roundtrip_and_reject(oracle, saber_tv):
    pk, sk, buf = saber_tv["pk"][None], saber_tv["sk"][None], saber_tv["buf"][None, :32]
    ct, ss = oracle.enc(3, pk, buf)
    assert (oracle.dec(3, ct, sk) == ss).all()
    bad = ct.copy()
    bad[0, 5] ^= 1
    rej = oracle.dec(3, bad, sk)
    z = sk[0, -32:].tobytes()
    exp = hashlib.sha3_256(z + hashlib.sha3_256(bad[0].tobytes()).digest()).digest()
    assert rej[0].tobytes() == exp
