"""Mixed-scheme, mixed-operation batches in one persistent launch: every request's output
must equal what the batched entry points produce for the same inputs (alone vs in the mix)."""
import numpy as np
import pytest
import torch

import dpcrypto_b200 as d

pytestmark = pytest.mark.gpu
SCHEMES = [d.FRODO976, d.LIGHTSABER, d.SABER, d.FIRESABER]


def _mixed_case(engine, per_kind, seed, form):
    """Requests: per scheme, per_kind keypairs, encaps and decaps (some tampered), shuffled."""
    rng = np.random.default_rng(seed)
    items, expect = [], []
    for scheme in SCHEMES:
        z = d.sizes(scheme)
        n = per_kind
        kc = torch.empty((3 * n, z["kp_coins"]), dtype=torch.uint8, device="cuda")
        ec = torch.empty((2 * n, z["enc_coins"]), dtype=torch.uint8, device="cuda")
        engine.coins(3 * n, z["kp_coins"], "kp", first=seed * 1000 + scheme * 100, out=kc)
        engine.coins(2 * n, z["enc_coins"], "enc", first=seed * 1000 + scheme * 100, out=ec)
        # reference results from the batched calls
        pk, sk = engine.keypair(scheme, kc, d.FORM_DP4A)
        ct, ss = engine.enc(scheme, pk[:2 * n], ec, d.FORM_DP4A)
        ct_dec = ct[n:].clone()
        ct_dec[::2, 3] ^= 1  # half of the decaps get a tampered ciphertext
        ss_dec = engine.dec(scheme, ct_dec, sk[n:2 * n], d.FORM_DP4A)
        torch.cuda.synchronize()
        for i in range(n):  # keypair requests on coins n..2n... use the third block of coins
            opk = torch.empty(z["pk"], dtype=torch.uint8, device="cuda")
            osk = torch.empty(z["sk"], dtype=torch.uint8, device="cuda")
            items.append((scheme, 0, kc[2 * n + i], None, opk, osk))
            expect.append(((opk, pk[2 * n + i]), (osk, sk[2 * n + i])))
        for i in range(n):
            oct_ = torch.empty(z["ct"], dtype=torch.uint8, device="cuda")
            oss = torch.empty(z["ss"], dtype=torch.uint8, device="cuda")
            items.append((scheme, 1, ec[i], pk[i], oct_, oss))
            expect.append(((oct_, ct[i]), (oss, ss[i])))
        for i in range(n):
            oss = torch.empty(z["ss"], dtype=torch.uint8, device="cuda")
            items.append((scheme, 2, ct_dec[i], sk[n + i], oss, None))
            expect.append(((oss, ss_dec[i]),))
    order = rng.permutation(len(items))
    return [items[k] for k in order], [expect[k] for k in order]


@pytest.mark.parametrize("form", [d.FORM_TC, d.FORM_DP4A, d.FORM_INT32])
def test_mixed_equals_batched(engine, form):
    items, expect = _mixed_case(engine, 5, 1, form)
    engine.mixed(items, form)
    engine.sync()
    torch.cuda.synchronize()
    for pairs in expect:
        for got, ref in pairs:
            assert torch.equal(got, ref)


def test_mixed_graph_replay(engine):
    items, expect = _mixed_case(engine, 3, 2, d.FORM_TC)
    g = engine.mixed_graph(items, d.FORM_TC)
    for _ in range(2):
        for pairs in expect:
            for got, _ in pairs:
                got.zero_()
        g.launch()
        torch.cuda.synchronize()
        engine.sync()
        for pairs in expect:
            for got, ref in pairs:
                assert torch.equal(got, ref)
    g.close()
