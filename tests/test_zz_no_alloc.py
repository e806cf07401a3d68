"""The allocation-free Saber encapsulation entry point against the regular one and the oracle.

dpkem_saber_enc_batch_static serves callers that may not call cudaMalloc on their
request path; its scratch is a fixed array inside the library.  Its output must equal
dpkem_enc_batch's, byte for byte, on consecutive calls that reuse that array, in every
product form, and a stride sample must equal the CPU oracle.  A call must leave the
device's free memory unchanged.  This file is collected last so a failure here cannot
hide the result of any other test.
"""
import ctypes

import numpy as np
import pytest
import torch

import dpcrypto_b200 as d

pytestmark = pytest.mark.gpu

FORMS = (d.FORM_TC, d.FORM_DP4A, d.FORM_INT32)


def _static_enc(scheme, form, pk, coins, stream=None, out=None):
    n = pk.shape[0]
    z = d.sizes(scheme)
    if out is None:
        out = (torch.zeros((n, z["ct"]), dtype=torch.uint8, device="cuda"),
               torch.zeros((n, 32), dtype=torch.uint8, device="cuda"))
    ct, ss = out
    lib = d.load()
    rc = lib.dpkem_saber_enc_batch_static(scheme, form, n, ctypes.c_void_p(coins.data_ptr()),
                                          ctypes.c_void_p(pk.data_ptr()), ctypes.c_void_p(ct.data_ptr()),
                                          ctypes.c_void_p(ss.data_ptr()),
                                          None if stream is None else ctypes.c_void_p(stream.cuda_stream))
    assert rc == 0, lib.dpkem_strerror(rc)
    assert lib.dpkem_last_status() == 0
    return ct, ss


@pytest.mark.parametrize("scheme", [d.LIGHTSABER, d.SABER, d.FIRESABER])
def test_static_matches_regular_on_two_calls(scheme, oracle):
    z = d.sizes(scheme)
    with d.Engine(0) as eng:
        for call, (n, first) in enumerate(((512, 0), (200, 4096))):
            kc = torch.empty((n, 96), dtype=torch.uint8, device="cuda")
            ec = torch.empty((n, 32), dtype=torch.uint8, device="cuda")
            eng.coins(n, 96, "kp", first=first, out=kc)
            eng.coins(n, 32, "enc", first=first, out=ec)
            pk, _ = eng.keypair(scheme, kc, d.FORM_TC)
            # the oracle on a stride sample of this call's instances
            idx = np.arange(call, n, 37)
            ct_o, ss_o = oracle.enc(scheme, pk.cpu().numpy()[idx], ec.cpu().numpy()[idx], threads=8)
            for form in FORMS:
                ct_ref, ss_ref = eng.enc(scheme, pk, ec, form)
                torch.cuda.synchronize()
                ct, ss = _static_enc(scheme, form, pk, ec)
                assert torch.equal(ct, ct_ref), (scheme, form, call)
                assert torch.equal(ss, ss_ref), (scheme, form, call)
                assert (ct.cpu().numpy()[idx] == ct_o).all(), (scheme, form, call)
                assert (ss.cpu().numpy()[idx] == ss_o).all(), (scheme, form, call)


def test_static_on_a_stream_allocates_nothing(oracle):
    """After a warm-up call (which may load the kernels), a second call on a caller's stream
    leaves the device's free memory exactly as it was, and gives the same bytes."""
    n, scheme = 300, d.SABER
    z = d.sizes(scheme)
    kc, ec = oracle.coins(n, 96, "kp", first=11), oracle.coins(n, 32, "enc", first=11)
    pk_o, _ = oracle.keypair(scheme, kc, threads=8)
    ct_o, ss_o = oracle.enc(scheme, pk_o, ec, threads=8)
    pk, coins = torch.from_numpy(pk_o).cuda(), torch.from_numpy(ec).cuda()
    outs = [(torch.zeros((n, z["ct"]), dtype=torch.uint8, device="cuda"),
             torch.zeros((n, 32), dtype=torch.uint8, device="cuda")) for _ in range(2)]
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    _static_enc(scheme, d.FORM_TC, pk, coins, stream=s, out=outs[0])
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    _static_enc(scheme, d.FORM_TC, pk, coins, stream=s, out=outs[1])
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
    for ct, ss in outs:
        assert (ct.cpu().numpy() == ct_o).all() and (ss.cpu().numpy() == ss_o).all()


def test_static_rejects_oversize_batch():
    n = 513
    buf = torch.zeros((n, 1472), dtype=torch.uint8, device="cuda")
    p = ctypes.c_void_p(buf.data_ptr())
    lib = d.load()
    rc = lib.dpkem_saber_enc_batch_static(d.SABER, d.FORM_TC, n, p, p, p, p, None)
    assert rc == d.kem.EINVAL
    assert lib.dpkem_last_status() == d.kem.EINVAL
