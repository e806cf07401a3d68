"""Oracle self-consistency: round trips and implicit rejection for every scheme."""
import hashlib

import numpy as np
import pytest


@pytest.mark.parametrize("scheme", [0, 2, 3, 4])
def test_roundtrip_and_reject(oracle, scheme):
    n = 4 if scheme == 0 else 32
    z = oracle.sizes(scheme)
    pk, sk = oracle.keypair(scheme, oracle.coins(n, z["kp_coins"], "kp"), threads=4)
    ct, ss = oracle.enc(scheme, pk, oracle.coins(n, z["enc_coins"], "enc"), threads=4)
    assert (oracle.dec(scheme, ct, sk, threads=4) == ss).all()
    bad = ct.copy()
    for i in range(n):
        bad[i, (i * 7919) % z["ct"]] ^= 1 << (i % 8)
    rej = oracle.dec(scheme, bad, sk, threads=4)
    assert (rej != ss).any(axis=1).all()
    if scheme == 0:  # implicit reject key = SHAKE256(ct || s)
        for i in range(n):
            assert rej[i].tobytes() == hashlib.shake_256(bad[i].tobytes() + sk[i, :24].tobytes()).digest(24)


def test_frodo_layout(oracle):
    pk, sk = oracle.keypair(0, oracle.coins(1, 64, "kp"))
    assert (sk[0, 24:24 + 15632] == pk[0]).all()
    assert sk[0, -24:].tobytes() == hashlib.shake_256(pk[0].tobytes()).digest(24)
    c = oracle.coins(1, 64, "kp")[0]
    assert pk[0, :16].tobytes() == hashlib.shake_256(c[48:64].tobytes()).digest(16)
    s_t = sk[0, 24 + 15632:24 + 15632 + 15616].view("<u2").astype(np.int16)
    assert s_t.min() >= -10 and s_t.max() <= 10


def test_frodo_sampler_table(oracle):
    # Exhaustive over all 16-bit inputs: output is +-k where k counts CDF entries below r >> 1.
    w = np.arange(65536, dtype=np.uint16)
    out = oracle.frodo_sample(w).astype(np.int16)
    cdf = np.array([5638, 15915, 23689, 28571, 31116, 32217, 32613, 32731, 32760, 32766])
    mag = (np.arange(65536)[:, None] >> 1 > cdf[None, :]).sum(1)
    sign = np.arange(65536) & 1
    assert (out == np.where(sign == 1, -mag, mag)).all()
