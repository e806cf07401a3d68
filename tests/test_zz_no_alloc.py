"""The allocation-free Saber encapsulation entry point against the regular one.

dpkem_saber_enc_batch_static serves callers that may not call cudaMalloc on their
request path; its scratch is a fixed array inside the library.  Its output must equal
dpkem_enc_batch's, byte for byte, on consecutive calls that reuse that array.  This file
is collected last so a failure here cannot hide the result of any other test.
"""
import ctypes

import numpy as np
import pytest
import torch

import dpcrypto_b200 as d

pytestmark = pytest.mark.gpu


def _static_enc(scheme, form, pk, coins):
    n = pk.shape[0]
    z = d.sizes(scheme)
    ct = torch.zeros((n, z["ct"]), dtype=torch.uint8, device="cuda")
    ss = torch.zeros((n, 32), dtype=torch.uint8, device="cuda")
    rc = d.load().dpkem_saber_enc_batch_static(scheme, form, n, ctypes.c_void_p(coins.data_ptr()),
                                               ctypes.c_void_p(pk.data_ptr()), ctypes.c_void_p(ct.data_ptr()),
                                               ctypes.c_void_p(ss.data_ptr()), None)
    assert rc == 0, d.load().dpkem_strerror(rc)
    return ct, ss


@pytest.mark.parametrize("scheme", [d.LIGHTSABER, d.SABER, d.FIRESABER])
def test_static_matches_regular_on_two_calls(scheme):
    z = d.sizes(scheme)
    with d.Engine(0) as eng:
        for call, (n, first) in enumerate(((512, 0), (200, 4096))):
            kc = torch.empty((n, 96), dtype=torch.uint8, device="cuda")
            ec = torch.empty((n, 32), dtype=torch.uint8, device="cuda")
            eng.coins(n, 96, "kp", first=first, out=kc)
            eng.coins(n, 32, "enc", first=first, out=ec)
            pk, _ = eng.keypair(scheme, kc, d.FORM_TC)
            for form in (d.FORM_TC, d.FORM_DP4A):
                ct_ref, ss_ref = eng.enc(scheme, pk, ec, form)
                torch.cuda.synchronize()
                ct, ss = _static_enc(scheme, form, pk, ec)
                assert torch.equal(ct, ct_ref), (scheme, form, call)
                assert torch.equal(ss, ss_ref), (scheme, form, call)


def test_static_rejects_oversize_batch():
    n = 513
    buf = torch.zeros((n, 1472), dtype=torch.uint8, device="cuda")
    p = ctypes.c_void_p(buf.data_ptr())
    rc = d.load().dpkem_saber_enc_batch_static(d.SABER, d.FORM_TC, n, p, p, p, p, None)
    assert rc == d.kem.EINVAL
