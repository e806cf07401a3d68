"""Pin the oracle's Keccak / SHA-3 / SHAKE against Python's hashlib (independent implementation)."""
import hashlib

import numpy as np
import pytest

LENGTHS = [0, 1, 7, 8, 71, 72, 73, 135, 136, 137, 167, 168, 169, 500, 15632, 15768]


@pytest.mark.parametrize("n", LENGTHS)
def test_sha3_and_shake(oracle, n):
    rng = np.random.default_rng(n)
    msg = rng.integers(0, 256, n, dtype=np.uint8).tobytes()
    assert oracle.sha3_256(msg) == hashlib.sha3_256(msg).digest()
    assert oracle.sha3_512(msg) == hashlib.sha3_512(msg).digest()
    for out in (16, 24, 48, 168, 1952, 31360):
        assert oracle.shake128(msg, out) == hashlib.shake_128(msg).digest(out)
        assert oracle.shake256(msg, out) == hashlib.shake_256(msg).digest(out)


def test_coins_stream(oracle):
    c = oracle.coins(5, 64, "kp", first=7)
    for i in range(5):
        ref = hashlib.shake_256(bytes(range(32)) + (7 + i).to_bytes(8, "little") + b"kp").digest(64)
        assert c[i].tobytes() == ref


def test_unrolled_permutation_equals_loop_form(oracle):
    """The sponge's unrolled Keccak-f (constant indices and rotations) against the loop form
    restated over the (x, y) grid, on random and edge states."""
    import numpy as np

    lib = oracle.lib()
    rng = np.random.default_rng(5)
    states = [np.zeros(25, np.uint64), np.full(25, np.uint64(0xFFFFFFFFFFFFFFFF), np.uint64)]
    states += [rng.integers(0, 2**63, size=25, dtype=np.uint64) * np.uint64(2) + np.uint64(k & 1) for k in range(300)]
    for st in states:
        a, b = st.copy(), st.copy()
        lib.oracle_keccak_f1600(a.ctypes.data)
        lib.oracle_keccak_f1600_plain(b.ctypes.data)
        assert (a == b).all()
