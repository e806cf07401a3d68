"""FrodoKEM batches under one key: A expanded once (dpkem_frodo_expand_a) against the oracle's
rows, and n encapsulations to one public key / n decapsulations with one secret key, with A
from memory or regenerated, in every product form, byte for byte against the oracle."""
import numpy as np
import pytest
import torch

import dpcrypto_b200 as d

pytestmark = pytest.mark.gpu
FORMS = [d.FORM_TC, d.FORM_DP4A, d.FORM_INT32]


def _tamper(ct):
    bad = ct.copy()
    for i in range(bad.shape[0]):
        bad[i, (i * 7919) % bad.shape[1]] ^= 1 << (i % 8)
    return bad


@pytest.mark.parametrize("scheme", [d.FRODO976, d.FRODO976AES])
def test_expand_a_matches_oracle_rows(engine, oracle, scheme):
    kc = oracle.coins(1, 64, "kp", first=314)
    pk, _ = oracle.keypair(scheme, kc)
    amat = engine.expand_a(scheme, torch.from_numpy(pk[0].copy()).cuda()).cpu().numpy().view(np.uint16)
    gen = oracle.frodo_gen_row if scheme == d.FRODO976 else oracle.frodo_gen_row_aes
    for i in (0, 1, 255, 256, 511, 974, 975):
        assert (amat[i] == gen(pk[0, :16].tobytes(), i)).all(), i


@pytest.mark.parametrize("form", FORMS)
@pytest.mark.parametrize("scheme", [d.FRODO976, d.FRODO976AES])
@pytest.mark.parametrize("with_a", [True, False])
def test_shared_key_enc_dec_match_oracle(engine, oracle, scheme, form, with_a):
    n = 9
    kc = oracle.coins(1, 64, "kp", first=271)
    pk, sk = oracle.keypair(scheme, kc)
    ec = oracle.coins(n, 24, "enc", first=271)
    pk_n, sk_n = np.repeat(pk, n, axis=0), np.repeat(sk, n, axis=0)
    ct_o, ss_o = oracle.enc(scheme, pk_n, ec, threads=8)
    bad = _tamper(ct_o)
    ssb_o = oracle.dec(scheme, bad, sk_n, threads=8)
    dpk, dsk = torch.from_numpy(pk[0].copy()).cuda(), torch.from_numpy(sk[0].copy()).cuda()
    amat = engine.expand_a(scheme, dpk) if with_a else None
    ct, ss = engine.enc_shared(scheme, dpk, torch.from_numpy(ec).cuda(), form, amat)
    torch.cuda.synchronize()
    assert (ct.cpu().numpy() == ct_o).all() and (ss.cpu().numpy() == ss_o).all()
    ss2 = engine.dec_shared(scheme, torch.from_numpy(ct_o).cuda(), dsk, form, amat)
    ss3 = engine.dec_shared(scheme, torch.from_numpy(bad).cuda(), dsk, form, amat)
    torch.cuda.synchronize()
    assert (ss2.cpu().numpy() == ss_o).all()
    assert (ss3.cpu().numpy() == ssb_o).all()


@pytest.mark.parametrize("scheme", [d.FRODO976, d.FRODO976AES])
def test_shared_key_gemm_groups_and_tampering(engine, oracle, scheme):
    """The tensor-core shared-key path (A in memory: the products as one GEMM over 16-instance
    groups) at a size with a partial last group; decaps ciphertexts tampered in B' (one
    instance in three), in C (one in three) or left intact, against the oracle and against the
    same batch with A regenerated per instance."""
    n = 37
    kc = oracle.coins(1, 64, "kp", first=977)
    pk, sk = oracle.keypair(scheme, kc)
    ec = oracle.coins(n, 24, "enc", first=977)
    pk_n, sk_n = np.repeat(pk, n, axis=0), np.repeat(sk, n, axis=0)
    ct_o, ss_o = oracle.enc(scheme, pk_n, ec, threads=8)
    bad = ct_o.copy()
    pkb = 2 * 976 * 8
    for i in range(n):
        if i % 3 == 0:
            bad[i, pkb + (13 * i) % 128] ^= 1 << (i % 8)
        elif i % 3 == 1:
            bad[i, (7919 * i) % pkb] ^= 1 << (i % 8)
    ssb_o = oracle.dec(scheme, bad, sk_n, threads=8)
    dpk, dsk = torch.from_numpy(pk[0].copy()).cuda(), torch.from_numpy(sk[0].copy()).cuda()
    amat = engine.expand_a(scheme, dpk)
    ct, ss = engine.enc_shared(scheme, dpk, torch.from_numpy(ec).cuda(), d.FORM_TC, amat)
    ssb = engine.dec_shared(scheme, torch.from_numpy(bad).cuda(), dsk, d.FORM_TC, amat)
    ssb_regen = engine.dec_shared(scheme, torch.from_numpy(bad).cuda(), dsk, d.FORM_TC, None)
    torch.cuda.synchronize()
    assert (ct.cpu().numpy() == ct_o).all() and (ss.cpu().numpy() == ss_o).all()
    assert (ssb.cpu().numpy() == ssb_o).all()
    assert torch.equal(ssb, ssb_regen)
    differs = (ssb_o != ss_o).any(axis=1)
    assert not differs[2::3].any() and differs[0::3].all() and differs[1::3].all()


def test_shared_key_gemm_2048(engine, oracle):
    """2,048 encapsulations to one key and their decapsulations through the tensor-core GEMM
    (the profiling case of gemm_kernel), equal to the per-instance path with A regenerated,
    and on a stride of instances to the oracle."""
    n = 2048
    kc = oracle.coins(1, 64, "kp", first=2048)
    pk, sk = oracle.keypair(d.FRODO976, kc)
    ec = oracle.coins(n, 24, "enc", first=2048)
    dpk, dsk = torch.from_numpy(pk[0].copy()).cuda(), torch.from_numpy(sk[0].copy()).cuda()
    dec = torch.from_numpy(ec).cuda()
    amat = engine.expand_a(d.FRODO976, dpk)
    ct, ss = engine.enc_shared(d.FRODO976, dpk, dec, d.FORM_TC, amat)
    ss2 = engine.dec_shared(d.FRODO976, ct, dsk, d.FORM_TC, amat)
    ct_r, ss_r = engine.enc_shared(d.FRODO976, dpk, dec, d.FORM_TC, None)
    torch.cuda.synchronize()
    assert torch.equal(ct, ct_r) and torch.equal(ss, ss_r) and torch.equal(ss2, ss)
    idx = np.arange(0, n, 97)
    ct_o, ss_o = oracle.enc(d.FRODO976, np.repeat(pk, len(idx), axis=0), ec[idx], threads=8)
    assert (ct.cpu().numpy()[idx] == ct_o).all() and (ss.cpu().numpy()[idx] == ss_o).all()
