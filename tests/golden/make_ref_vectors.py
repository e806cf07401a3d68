"""Generate tests/golden/ref_vectors.npz: known-answer vectors computed by the reference's
own kernels.

oracle/ref builds the reference's CUDA sources (FrodoKEM976-GPU/src, SABER-GPU/src) as host
C++ through a small CUDA emulation layer into oracle/_ref/libref_*.so, and assembles them
into keypair / encaps / decaps at one instance per call (oracle/ref/frodo_ref.cpp and
saber_ref.cpp list the few steps that are glue and why).  This script runs them on seeded
coins and stores, per scheme: the coins, SHA-256 digests of pk, sk and ct (every byte is
pinned, the fixture stays small), the encapsulated secret, and the secret that decaps gives
for the ciphertext and for a tampered copy of it (bit (i mod 8) of byte (7919 i mod |ct|)).

Run where the reference tree is present (it is not needed afterwards):
    make -C oracle/ref REF=<reference tree>
    python tests/golden/make_ref_vectors.py
"""
import ctypes
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402  (seeded coin stream only)

REF = os.path.join(ROOT, "oracle", "_ref")
# scheme -> (library, symbol prefix, pk, sk, ct, ss, kp coins, enc coins, instances)
SCHEMES = {
    0: ("libref_frodo.so", "ref_frodo", 15632, 31296, 15744, 24, 64, 24, 8),
    2: ("libref_saber2.so", "ref_saber2", 672, 1568, 736, 32, 96, 32, 24),
    3: ("libref_saber3.so", "ref_saber3", 992, 2304, 1088, 32, 96, 32, 24),
    4: ("libref_saber4.so", "ref_saber4", 1312, 3040, 1472, 32, 96, 32, 24),
}


def digest(a: np.ndarray) -> np.ndarray:
    return np.frombuffer(hashlib.sha256(a.tobytes()).digest(), np.uint8)


def tamper(ct: np.ndarray, i: int) -> np.ndarray:
    bad = ct.copy()
    bad[(i * 7919) % bad.size] ^= 1 << (i % 8)
    return bad


def coins(n: int, length: int, tag: str) -> np.ndarray:
    """Seeded coins; the last two instances are the all-zero and all-0xFF edge cases."""
    c = O.coins(n, length, tag, first=1000)
    c[-2] = 0
    c[-1] = 0xFF
    return np.ascontiguousarray(c)


def run(scheme: int) -> dict:
    so, pre, npk, nsk, nct, nss, nkc, nec, n = SCHEMES[scheme]
    lib = ctypes.CDLL(os.path.join(REF, so))
    kp, enc, dec = (getattr(lib, f"{pre}_{op}") for op in ("keypair", "enc", "dec"))
    for f in (kp, enc, dec):
        f.restype = ctypes.c_int

    def ptr(a):
        return ctypes.c_void_p(a.ctypes.data)

    kc, ec = coins(n, nkc, "ref-kp"), coins(n, nec, "ref-enc")
    out = {k: [] for k in ("pk", "sk", "ct", "ss", "ss_dec", "ss_tampered")}
    for i in range(n):
        kci, eci = kc[i].copy(), ec[i].copy()
        pk, sk = np.zeros(npk, np.uint8), np.zeros(nsk, np.uint8)
        ct, ss = np.zeros(nct, np.uint8), np.zeros(nss, np.uint8)
        ss_dec, ss_bad = np.zeros(nss, np.uint8), np.zeros(nss, np.uint8)
        bad = None
        assert kp(ptr(pk), ptr(sk), ptr(kci)) == 0
        assert enc(ptr(ct), ptr(ss), ptr(pk), ptr(eci)) == 0
        assert dec(ptr(ss_dec), ptr(ct), ptr(sk)) == 0
        bad = tamper(ct, i)
        assert dec(ptr(ss_bad), ptr(bad), ptr(sk)) == 0
        assert (ss_dec == ss).all() and (ss_bad != ss).any()
        for k, v in (("pk", digest(pk)), ("sk", digest(sk)), ("ct", digest(ct)), ("ss", ss), ("ss_dec", ss_dec),
                     ("ss_tampered", ss_bad)):
            out[k].append(v)
    res = {f"s{scheme}_{k}": np.stack(v) for k, v in out.items()}
    res[f"s{scheme}_kp_coins"], res[f"s{scheme}_enc_coins"] = kc, ec
    return res


def main() -> None:
    O.build()
    arrays = {}
    for scheme in SCHEMES:
        arrays.update(run(scheme))
        print("scheme", scheme, "done", flush=True)
    dst = os.path.join(HERE, "ref_vectors.npz")
    np.savez_compressed(dst, **arrays)
    print("wrote", dst, os.path.getsize(dst), "bytes")


if __name__ == "__main__":
    main()
