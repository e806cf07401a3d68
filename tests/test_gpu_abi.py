"""C-ABI behaviour on the GPU: status codes, device-pointer mode, chunking under a small
HBM budget, device coin stream, and the reference-named shims."""
import numpy as np
import pytest
import torch

import dpcrypto_b200 as d

pytestmark = pytest.mark.gpu


def test_status_codes(engine, oracle):
    kc = oracle.coins(2, 96, "kp")
    with pytest.raises(d.DpkemError) as e:
        engine.keypair(d.SABER, kc, 3)  # no form 3
    assert e.value.status == d.kem.EINVAL
    with pytest.raises(d.DpkemError) as e:
        engine.keypair(7, kc, d.FORM_TC)
    assert e.value.status == d.kem.EINVAL
    with pytest.raises(ValueError):
        engine.keypair(d.SABER, kc[:, :95].copy(), d.FORM_TC)
    empty = np.zeros((0, 96), np.uint8)
    pk, sk = engine.keypair(d.SABER, empty, d.FORM_TC)
    assert pk.shape == (0, 992) and sk.shape == (0, 2304)


def test_device_coins_match_oracle(engine, oracle):
    for length, tag in ((64, "kp"), (24, "enc"), (96, "kp"), (32, "enc"), (5, "x")):
        host = engine.coins(37, length, tag, first=3)
        assert (host == oracle.coins(37, length, tag, first=3)).all()
        dev = torch.empty((37, length), dtype=torch.uint8, device="cuda")
        engine.coins(37, length, tag, first=3, out=dev)
        torch.cuda.synchronize()
        assert (dev.cpu().numpy() == host).all()


@pytest.mark.parametrize("scheme", [d.FRODO976, d.SABER])
def test_device_pointer_mode(engine, oracle, scheme):
    z = d.sizes(scheme)
    n = 40
    kc = torch.from_numpy(oracle.coins(n, z["kp_coins"], "kp")).cuda()
    ec = torch.from_numpy(oracle.coins(n, z["enc_coins"], "enc")).cuda()
    pk, sk = engine.keypair(scheme, kc, d.FORM_TC)
    ct, ss = engine.enc(scheme, pk, ec, d.FORM_TC)
    ss2 = engine.dec(scheme, ct, sk, d.FORM_TC)
    engine.sync(ctypes_stream(torch.cuda.current_stream()))
    assert torch.equal(ss, ss2)
    pk_h, _ = engine.keypair(scheme, kc.cpu().numpy(), d.FORM_DP4A)
    assert (pk.cpu().numpy() == pk_h).all()


def ctypes_stream(s):
    import ctypes

    return ctypes.c_void_p(s.cuda_stream)


@pytest.mark.parametrize("scheme", [d.FRODO976, d.SABER])
def test_chunking_under_small_budget(oracle, scheme):
    z = d.sizes(scheme)
    budget = (2 << 20) if scheme == d.FRODO976 else (256 << 10)
    with d.Engine(0, hbm_budget=budget) as small:
        assert small.max_chunk(scheme) < 40
        n = 40
        kc, ec = oracle.coins(n, z["kp_coins"], "kp"), oracle.coins(n, z["enc_coins"], "enc")
        pk, sk = small.keypair(scheme, kc, d.FORM_TC)
        ct, ss = small.enc(scheme, pk, ec, d.FORM_TC)
        assert (small.dec(scheme, ct, sk, d.FORM_TC) == ss).all()
    with d.Engine(0) as big:
        pk2, _ = big.keypair(scheme, kc, d.FORM_TC)
        assert (pk2 == pk).all()


def test_reference_named_shims(oracle):
    n = 4
    d.set_compat(batch=n, saber_level=3, form=d.FORM_TC)
    pk, sk = np.zeros((n, 15632), np.uint8), np.zeros((n, 31296), np.uint8)
    d.frodoKEMKeypair(pk, sk)
    pk_o, sk_o = oracle.keypair(0, oracle.coins(n, 64, "kp"), threads=4)
    assert (pk == pk_o).all() and (sk == sk_o).all()
    ct, ssb, ssa = np.zeros((n, 15744), np.uint8), np.zeros((n, 24), np.uint8), np.zeros((n, 24), np.uint8)
    d.frodoKEMEncap(ct, ssb, pk)
    d.frodoKEMDecap(ssa, ct, sk)
    assert (ssa == ssb).all()
    spk, ssk = oracle.keypair(3, oracle.coins(n, 96, "kp"), threads=4)
    # the shims draw their encaps coins from the same seeded stream (instances 0..n-1, "enc")
    c_o, k_o = oracle.enc(3, spk, oracle.coins(n, 32, "enc"), threads=4)
    for mode in (0, 1, 2):  # the reference's modes: 0 dp4a, 1 INT32 schoolbook, 2 tensor cores
        k_enc, c = np.zeros((n, 32), np.uint8), np.zeros((n, 1088), np.uint8)
        d.saber_enc(mode, k_enc, spk, c)
        assert (c == c_o).all() and (k_enc == k_o).all(), mode
        k_dec = np.zeros((n, 32), np.uint8)
        d.saber_dec(mode, c, spk, ssk, k_dec)
        assert (k_dec == k_o).all(), mode
    # a mode byte the reference does not define is rejected and nothing is written
    for mode in (3, 7, 255):
        k_enc, c = np.zeros((n, 32), np.uint8), np.zeros((n, 1088), np.uint8)
        with pytest.raises(d.DpkemError) as e:
            d.saber_enc(mode, k_enc, spk, c)
        assert e.value.status == d.kem.EINVAL and not c.any() and not k_enc.any()
        with pytest.raises(d.DpkemError) as e:
            d.saber_dec(mode, c_o, spk, ssk, k_enc)
        assert e.value.status == d.kem.EINVAL and not k_enc.any()
    d.set_compat(batch=768)


@pytest.mark.parametrize("scheme,n", [(d.SABER, 1100), (d.FRODO976, 600), (d.FRODO976, 1100)])
def test_host_pipeline_matches_device_mode(engine, oracle, scheme, n):
    """Host-mode batches of several chunks run as a copy/compute pipeline, one stream per
    chunk (600: two equal chunks; 1100: four, the first and last a quarter of the others)."""
    z = d.sizes(scheme)
    kc, ec = oracle.coins(n, z["kp_coins"], "kp", first=77), oracle.coins(n, z["enc_coins"], "enc", first=77)
    pk, sk = engine.keypair(scheme, kc, d.FORM_TC)
    ct, ss = engine.enc(scheme, pk, ec, d.FORM_TC)
    ss2 = engine.dec(scheme, ct, sk, d.FORM_TC)
    dpk, dsk = engine.keypair(scheme, torch.from_numpy(kc).cuda(), d.FORM_TC)
    dct, dss = engine.enc(scheme, dpk, torch.from_numpy(ec).cuda(), d.FORM_TC)
    torch.cuda.synchronize()
    assert (dpk.cpu().numpy() == pk).all() and (dsk.cpu().numpy() == sk).all()
    assert (dct.cpu().numpy() == ct).all() and (dss.cpu().numpy() == ss).all()
    assert (ss2 == ss).all()


@pytest.mark.parametrize("which", [0, 1])
def test_bounded_wait_expiry(engine, oracle, which):
    """A device wait that nothing can satisfy expires after its limit and comes back as
    DPKEM_ETIMEOUT (no trap, no hang); the context keeps working afterwards."""
    assert engine._lib.dpkem_selftest_timeout(engine._h, which) == d.kem.ETIMEOUT
    kc, ec = oracle.coins(3, 96, "kp", first=9), oracle.coins(3, 32, "enc", first=9)
    pk, sk = engine.keypair(d.SABER, kc, d.FORM_TC)
    pk_o, sk_o = oracle.keypair(3, kc)
    assert (pk == pk_o).all() and (sk == sk_o).all()
    z = d.sizes(d.SABER)
    items, outs = [], []
    for i in range(3):
        oct_ = torch.empty(z["ct"], dtype=torch.uint8, device="cuda")
        oss = torch.empty(z["ss"], dtype=torch.uint8, device="cuda")
        items.append((d.SABER, 1, torch.from_numpy(ec[i].copy()).cuda(), torch.from_numpy(pk[i].copy()).cuda(),
                      oct_, oss))
        outs.append((oct_, oss))
    engine.mixed(items, d.FORM_TC)
    engine.sync()
    ct_o, ss_o = oracle.enc(3, pk_o, ec)
    for i, (c, s) in enumerate(outs):
        assert (c.cpu().numpy() == ct_o[i]).all() and (s.cpu().numpy() == ss_o[i]).all()


def test_i8_mma_peak_probe(engine):
    """The tensor-peak probe runs (valid descriptors, bounded wait) and reports a plausible
    int8 MAC rate for a B200-class GPU (dense int8 is ~2 P MAC/s)."""
    macs = engine.probe_i8_mma_peak()
    assert 1e14 < macs < 1e16


@pytest.mark.parametrize("chunks,prio", [(2, 0), (8, 1), (16, 1)])
def test_host_pipeline_depths(engine, chunks, prio):
    """Host-buffer batches split into up to 16 pipelined chunks (one stream each, with or
    without descending priorities) give the device-pointer results on every instance."""
    from dpcrypto_b200 import kem

    for scheme, n in ((d.SABER, 4096), (d.FRODO976, 4096)):
        z = d.sizes(scheme)
        kc = torch.empty((n, z["kp_coins"]), dtype=torch.uint8, device="cuda")
        ec = torch.empty((n, z["enc_coins"]), dtype=torch.uint8, device="cuda")
        engine.coins(n, z["kp_coins"], "pipe-kp", first=chunks, out=kc)
        engine.coins(n, z["enc_coins"], "pipe-enc", first=chunks, out=ec)
        pk, sk = engine.keypair(scheme, kc, d.FORM_TC)
        ct, ss = engine.enc(scheme, pk, ec, d.FORM_TC)
        ss2 = engine.dec(scheme, ct, sk, d.FORM_TC)
        torch.cuda.synchronize()
        with kem.knobs(pipe_chunks=chunks, pipe_priority=prio):
            h_ct, h_ss = engine.enc(scheme, pk.cpu().numpy(), ec.cpu().numpy(), d.FORM_TC)
            h_ss2 = engine.dec(scheme, h_ct, sk.cpu().numpy(), d.FORM_TC)
        assert (h_ct == ct.cpu().numpy()).all() and (h_ss == ss.cpu().numpy()).all()
        assert (h_ss2 == ss2.cpu().numpy()).all() and (h_ss2 == h_ss).all()
