"""Every product form on the GPU against the known answers computed by the reference's own
kernels (tests/golden/ref_vectors.npz, made by tests/golden/make_ref_vectors.py): keypair,
encaps and decaps (valid and tampered ciphertexts) of FrodoKEM-976 and Saber l = 2, 3, 4,
through the C ABI, every byte compared (pk, sk and ct through SHA-256 digests)."""
import hashlib
import os

import numpy as np
import pytest

import dpcrypto_b200 as d

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
FORMS = [d.FORM_TC, d.FORM_DP4A, d.FORM_INT32]


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


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("scheme", [d.FRODO976, d.LIGHTSABER, d.SABER, d.FIRESABER])
def test_gpu_matches_reference_vectors(engine, vectors, scheme, form):
    v = {k[len(f"s{scheme}_"):]: a for k, a in vectors.items() if k.startswith(f"s{scheme}_")}
    pk, sk = engine.keypair(scheme, v["kp_coins"], form)
    assert (_digests(pk) == v["pk"]).all() and (_digests(sk) == v["sk"]).all()
    ct, ss = engine.enc(scheme, pk, v["enc_coins"], form)
    assert (_digests(ct) == v["ct"]).all() and (ss == v["ss"]).all()
    assert (engine.dec(scheme, ct, sk, form) == v["ss_dec"]).all()
    assert (engine.dec(scheme, _tamper(ct), sk, form) == v["ss_tampered"]).all()
