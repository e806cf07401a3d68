"""The oracle's AES-128 (FIPS 197 restated) and FrodoKEM-976-AES matrix rows, pinned to
an independent AES: Python's `cryptography` package (OpenSSL's AES-ECB)."""
import struct

import numpy as np
import pytest

cryptography = pytest.importorskip("cryptography")
from cryptography.hazmat.primitives.ciphers import Cipher, algorithms, modes  # noqa: E402


def _ecb(key: bytes, data: bytes) -> bytes:
    e = Cipher(algorithms.AES(key), modes.ECB()).encryptor()
    return e.update(data) + e.finalize()


def test_aes128_matches_cryptography(oracle):
    rng = np.random.default_rng(0)
    for _ in range(20):
        key = rng.integers(0, 256, 16, dtype=np.uint8).tobytes()
        data = rng.integers(0, 256, 16 * 33, dtype=np.uint8).tobytes()
        assert oracle.aes128_ecb(key, data) == _ecb(key, data)
    for key in (bytes(16), bytes([0xFF]) * 16):  # edge keys, all-zero and all-one blocks
        data = bytes(16) + bytes([0xFF]) * 16
        assert oracle.aes128_ecb(key, data) == _ecb(key, data)


@pytest.mark.parametrize("i", [0, 1, 255, 256, 975])
def test_frodo_aes_row_matches_cryptography(oracle, i):
    seed = bytes(range(7, 23))
    blocks = b"".join(struct.pack("<HH", i, j) + bytes(12) for j in range(0, 976, 8))
    want = np.frombuffer(_ecb(seed, blocks), "<u2")
    assert (oracle.frodo_gen_row_aes(seed, i) == want).all()


def test_frodo_aes_roundtrip(oracle):
    n = 2
    kc, ec = oracle.coins(n, 64, "kp", first=3), oracle.coins(n, 24, "enc", first=3)
    pk, sk = oracle.keypair(oracle.FRODO_AES, kc, threads=2)
    pk_s, _ = oracle.keypair(oracle.FRODO, kc, threads=2)
    assert (pk[:, :16] == pk_s[:, :16]).all() and not (pk[:, 16:] == pk_s[:, 16:]).all()  # same seedA, other A
    ct, ss = oracle.enc(oracle.FRODO_AES, pk, ec, threads=2)
    assert (oracle.dec(oracle.FRODO_AES, ct, sk, threads=2) == ss).all()
    bad = ct.copy()
    bad[:, 100] ^= 1
    rej = oracle.dec(oracle.FRODO_AES, bad, sk, threads=2)
    assert not (rej == ss).all(axis=1).any()
