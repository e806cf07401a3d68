"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, __graft_entry__.smoke() and the
CPU-baseline legs of bench.py, always as the checker or the timed CPU baseline;
the product (dpcrypto_b200) never imports this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_NATIVE_PATH = os.path.join(_HERE, "_build", "native", "liboracle.so")
_lib = None
_native = False

FRODO = 0
FRODO_AES = 1
SABER_LEVELS = (2, 3, 4)
FRODO_SIZES = dict(pk=15632, sk=31296, ct=15744, ss=24, kp_coins=64, enc_coins=24)


def build() -> str:
    """Compile liboracle.so with the committed Makefile (gcc only)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def build_ref() -> None:
    """Build oracle/_ref (the reference's own kernels as host C++, oracle/ref/Makefile) when
    the reference tree is on this machine; a no-op elsewhere.  Checker code only."""
    subprocess.run(["make", "-s", "-C", os.path.join(_HERE, "ref")], check=True)


def use_native() -> str:
    """Switch this process to the CPU-baseline build of the oracle: the same sources compiled
    with -march=native on (and for) this machine, built here on first use.  Call before the
    first oracle call; the portable build stays the one the tests check."""
    global _native
    if _lib is not None and not _native:
        raise RuntimeError("use_native() must come before the first oracle call")
    subprocess.run(["make", "-s", "-C", _HERE, "native"], check=True)
    _native = True
    return _NATIVE_PATH


def lib():
    global _lib
    if _lib is None:
        path = _NATIVE_PATH if _native else _LIB_PATH
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        u8p = ctypes.c_void_p
        for name, args in {
            "oracle_keccak_f1600": [u8p],
            "oracle_keccak_f1600_plain": [u8p],
            "oracle_shake128": [u8p, ctypes.c_size_t, u8p, ctypes.c_size_t],
            "oracle_shake256": [u8p, ctypes.c_size_t, u8p, ctypes.c_size_t],
            "oracle_sha3_256": [u8p, u8p, ctypes.c_size_t],
            "oracle_sha3_512": [u8p, u8p, ctypes.c_size_t],
            "oracle_coins_batch": [u8p, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_size_t, ctypes.c_char_p],
            "oracle_frodo_keypair": [u8p, u8p, u8p],
            "oracle_frodo_enc": [u8p, u8p, u8p, u8p],
            "oracle_frodo_dec": [u8p, u8p, u8p],
            "oracle_frodo_gen_row": [u8p, u8p, ctypes.c_int],
            "oracle_frodo_gen_row_aes": [u8p, u8p, ctypes.c_int],
            "oracle_aes128_ecb": [u8p, u8p, ctypes.c_size_t, u8p],
            "oracle_frodo_sample": [u8p, ctypes.c_size_t],
            "oracle_saber_sizes": [ctypes.c_int] + [ctypes.POINTER(ctypes.c_size_t)] * 4,
            "oracle_saber_keypair": [ctypes.c_int, u8p, u8p, u8p],
            "oracle_saber_enc": [ctypes.c_int, u8p, u8p, u8p, u8p],
            "oracle_saber_dec": [ctypes.c_int, u8p, u8p, u8p],
            "oracle_saber_genmatrix": [ctypes.c_int, u8p, u8p],
            "oracle_saber_gensecret": [ctypes.c_int, u8p, u8p],
            "oracle_saber_matvec": [ctypes.c_int, u8p, u8p, u8p, ctypes.c_int],
            "oracle_batch": [ctypes.c_int, ctypes.c_int, ctypes.c_size_t, ctypes.c_int, u8p, u8p, u8p, u8p],
        }.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = ctypes.c_int if name not in ("oracle_keccak_f1600", "oracle_keccak_f1600_plain",
                                                     "oracle_shake128", "oracle_shake256", "oracle_sha3_256",
                                                     "oracle_sha3_512", "oracle_coins_batch",
                                                     "oracle_frodo_gen_row", "oracle_frodo_sample",
                                                     "oracle_frodo_gen_row_aes", "oracle_aes128_ecb",
                                                     "oracle_saber_genmatrix", "oracle_saber_gensecret",
                                                     "oracle_saber_matvec") else None
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return ctypes.c_void_p(a.ctypes.data)


def _u8(b) -> np.ndarray:
    return np.ascontiguousarray(np.frombuffer(bytes(b), dtype=np.uint8) if not isinstance(b, np.ndarray) else b,
                                dtype=np.uint8)


def shake128(data: bytes, n: int) -> bytes:
    out = np.zeros(n, np.uint8)
    src = _u8(data)
    lib().oracle_shake128(_p(out), n, _p(src) if src.size else None, src.size)
    return out.tobytes()


def shake256(data: bytes, n: int) -> bytes:
    out = np.zeros(n, np.uint8)
    src = _u8(data)
    lib().oracle_shake256(_p(out), n, _p(src) if src.size else None, src.size)
    return out.tobytes()


def sha3_256(data: bytes) -> bytes:
    out = np.zeros(32, np.uint8)
    src = _u8(data)
    lib().oracle_sha3_256(_p(out), _p(src) if src.size else None, src.size)
    return out.tobytes()


def sha3_512(data: bytes) -> bytes:
    out = np.zeros(64, np.uint8)
    src = _u8(data)
    lib().oracle_sha3_512(_p(out), _p(src) if src.size else None, src.size)
    return out.tobytes()


def coins(count: int, length: int, tag: str, first: int = 0) -> np.ndarray:
    """Seeded synthetic coins: row i = SHAKE256(00..1F || LE64(first+i) || tag, length)."""
    out = np.zeros((count, length), np.uint8)
    if count:
        lib().oracle_coins_batch(_p(out), length, first, count, tag.encode())
    return out


def sizes(scheme: int) -> dict:
    if scheme in (FRODO, FRODO_AES):
        return dict(FRODO_SIZES)
    pk, sk, ct, ss = (ctypes.c_size_t() for _ in range(4))
    if lib().oracle_saber_sizes(scheme, ctypes.byref(pk), ctypes.byref(sk), ctypes.byref(ct), ctypes.byref(ss)):
        raise ValueError(f"unknown Saber level {scheme}")
    return dict(pk=pk.value, sk=sk.value, ct=ct.value, ss=ss.value, kp_coins=96, enc_coins=32)


def keypair(scheme: int, kp_coins: np.ndarray, threads: int = 1):
    z = sizes(scheme)
    kp_coins = np.ascontiguousarray(kp_coins, np.uint8).reshape(-1, z["kp_coins"])
    n = kp_coins.shape[0]
    pk = np.zeros((n, z["pk"]), np.uint8)
    sk = np.zeros((n, z["sk"]), np.uint8)
    rc = lib().oracle_batch(scheme, 0, n, threads, _p(pk), _p(sk), _p(kp_coins), None)
    assert rc == 0
    return pk, sk


def enc(scheme: int, pk: np.ndarray, enc_coins: np.ndarray, threads: int = 1):
    z = sizes(scheme)
    pk = np.ascontiguousarray(pk, np.uint8).reshape(-1, z["pk"])
    enc_coins = np.ascontiguousarray(enc_coins, np.uint8).reshape(-1, z["enc_coins"])
    n = pk.shape[0]
    ct = np.zeros((n, z["ct"]), np.uint8)
    ss = np.zeros((n, z["ss"]), np.uint8)
    rc = lib().oracle_batch(scheme, 1, n, threads, _p(ct), _p(ss), _p(pk), _p(enc_coins))
    assert rc == 0
    return ct, ss


def dec(scheme: int, ct: np.ndarray, sk: np.ndarray, threads: int = 1):
    z = sizes(scheme)
    ct = np.ascontiguousarray(ct, np.uint8).reshape(-1, z["ct"])
    sk = np.ascontiguousarray(sk, np.uint8).reshape(-1, z["sk"])
    n = ct.shape[0]
    ss = np.zeros((n, z["ss"]), np.uint8)
    rc = lib().oracle_batch(scheme, 2, n, threads, _p(ss), None, _p(ct), _p(sk))
    assert rc == 0
    return ss


def frodo_gen_row(seed_a: bytes, i: int) -> np.ndarray:
    row = np.zeros(976, np.uint16)
    s = _u8(seed_a)
    lib().oracle_frodo_gen_row(_p(row), _p(s), i)
    return row


def frodo_gen_row_aes(seed_a: bytes, i: int) -> np.ndarray:
    row = np.zeros(976, np.uint16)
    s = _u8(seed_a)
    lib().oracle_frodo_gen_row_aes(_p(row), _p(s), i)
    return row


def aes128_ecb(key: bytes, data: bytes) -> bytes:
    """AES-128 ECB encryption of whole 16-byte blocks (oracle restatement of FIPS 197)."""
    if len(key) != 16 or len(data) % 16:
        raise ValueError("AES-128 ECB needs a 16-byte key and whole blocks")
    src, out, k = _u8(data), np.zeros(len(data), np.uint8), _u8(key)
    lib().oracle_aes128_ecb(_p(out), _p(src), len(data) // 16, _p(k))
    return out.tobytes()


def frodo_sample(words: np.ndarray) -> np.ndarray:
    w = np.ascontiguousarray(words, np.uint16).copy()
    lib().oracle_frodo_sample(_p(w), w.size)
    return w


def saber_genmatrix(level: int, seed: bytes) -> np.ndarray:
    a = np.zeros(level * level * 256, np.uint16)
    s = _u8(seed)
    lib().oracle_saber_genmatrix(level, _p(a), _p(s))
    return a


def saber_gensecret(level: int, seed: bytes) -> np.ndarray:
    out = np.zeros(level * 256, np.uint16)
    s = _u8(seed)
    lib().oracle_saber_gensecret(level, _p(out), _p(s))
    return out


def saber_matvec(level: int, a: np.ndarray, s: np.ndarray, transpose: bool) -> np.ndarray:
    res = np.zeros(level * 256, np.uint16)
    a = np.ascontiguousarray(a, np.uint16)
    s = np.ascontiguousarray(s, np.uint16)
    lib().oracle_saber_matvec(level, _p(res), _p(a), _p(s), int(transpose))
    return res
