"""The oracle pinned to the reference's own code.

tests/golden/ref_vectors.npz holds known answers computed by the reference's kernels
(FrodoKEM976-GPU/src, SABER-GPU/src built as host C++ by oracle/ref into oracle/_ref and
assembled at one instance per call; tests/golden/make_ref_vectors.py).  The oracle must
reproduce every byte (pk, sk and ct through SHA-256 digests, the shared secrets directly)
for FrodoKEM-976 and all three Saber levels, including the reject path and the all-zero and
all-0xFF coins.  Where oracle/_ref has been built (a machine with the reference tree), the
reference code is also run live against the oracle on fresh coins.
"""
import ctypes
import hashlib
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
SCHEMES = [0, 2, 3, 4]
LIBS = {0: ("libref_frodo.so", "ref_frodo"), 2: ("libref_saber2.so", "ref_saber2"),
        3: ("libref_saber3.so", "ref_saber3"), 4: ("libref_saber4.so", "ref_saber4")}


@pytest.fixture(scope="module")
def vectors():
    return dict(np.load(os.path.join(ROOT, "tests", "golden", "ref_vectors.npz")))


def _digests(a):
    return np.stack([np.frombuffer(hashlib.sha256(r.tobytes()).digest(), np.uint8) for r in a])


def _tamper(ct):
    bad = ct.copy()
    for i in range(bad.shape[0]):
        bad[i, (i * 7919) % bad.shape[1]] ^= 1 << (i % 8)
    return bad


@pytest.mark.parametrize("scheme", SCHEMES)
def test_oracle_matches_reference_vectors(oracle, vectors, scheme):
    v = {k[len(f"s{scheme}_"):]: a for k, a in vectors.items() if k.startswith(f"s{scheme}_")}
    pk, sk = oracle.keypair(scheme, v["kp_coins"], threads=8)
    assert (_digests(pk) == v["pk"]).all() and (_digests(sk) == v["sk"]).all()
    ct, ss = oracle.enc(scheme, pk, v["enc_coins"], threads=8)
    assert (_digests(ct) == v["ct"]).all() and (ss == v["ss"]).all()
    assert (oracle.dec(scheme, ct, sk, threads=8) == v["ss_dec"]).all()
    assert (oracle.dec(scheme, _tamper(ct), sk, threads=8) == v["ss_tampered"]).all()


def _lib(scheme):
    path = os.path.join(REF, LIBS[scheme][0])
    if not os.path.exists(path):
        pytest.skip("oracle/_ref not built (the reference tree is not on this machine)")
    return ctypes.CDLL(path), LIBS[scheme][1]


@pytest.mark.parametrize("scheme", SCHEMES)
def test_reference_code_live_against_oracle(oracle, scheme):
    lib, pre = _lib(scheme)
    z = oracle.sizes(scheme)
    n = 2 if scheme == 0 else 6
    kc, ec = oracle.coins(n, z["kp_coins"], "live-kp", first=7), oracle.coins(n, z["enc_coins"], "live-enc", first=7)
    pk_o, sk_o = oracle.keypair(scheme, kc, threads=8)
    ct_o, ss_o = oracle.enc(scheme, pk_o, ec, threads=8)
    for i in range(n):
        kci, eci = kc[i].copy(), ec[i].copy()
        pk, sk = np.zeros(z["pk"], np.uint8), np.zeros(z["sk"], np.uint8)
        ct, ss, ss2 = np.zeros(z["ct"], np.uint8), np.zeros(z["ss"], np.uint8), np.zeros(z["ss"], np.uint8)
        p = lambda a: ctypes.c_void_p(a.ctypes.data)  # noqa: E731
        assert getattr(lib, pre + "_keypair")(p(pk), p(sk), p(kci)) == 0
        assert getattr(lib, pre + "_enc")(p(ct), p(ss), p(pk), p(eci)) == 0
        assert getattr(lib, pre + "_dec")(p(ss2), p(ct), p(sk)) == 0
        assert (pk == pk_o[i]).all() and (sk == sk_o[i]).all()
        assert (ct == ct_o[i]).all() and (ss == ss_o[i]).all() and (ss2 == ss).all()


def test_reference_ct_verify_defect():
    """Records a reference defect that the harness (and this library) do not reproduce:
    ct_verify_gpu (FrodoKEM976-GPU/src/util.cu:193-207) reduces the OR of the differences
    with -(int16_t)r >> 15, which is 0 ("equal") whenever bit 15 of that OR is set, so the
    reference's decaps accepts such ciphertexts.  The specification's compare says "differ"."""
    lib, _ = _lib(0)
    f = lib.ref_frodo_ct_verify_raw
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t]
    a = np.zeros(64, np.uint16)
    for diff, said in ((0x0000, 0), (0x0001, -1), (0x7FFF, -1), (0x8000, 1), (0xFFFF, 0)):
        b = a.copy()
        b[5] = diff
        assert f(a.ctypes.data, b.ctypes.data, a.size) == said, hex(diff)
