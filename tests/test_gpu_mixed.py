"""Mixed-scheme, mixed-operation batches in one persistent launch: every request's output
must equal what the batched entry points produce for the same inputs (alone vs in the mix)."""
import numpy as np
import pytest
import torch

import dpcrypto_b200 as d

pytestmark = pytest.mark.gpu
SCHEMES = [d.FRODO976, d.FRODO976AES, d.LIGHTSABER, d.SABER, d.FIRESABER]


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


def _host_coins(key, index, tag, length):
    import hashlib
    import struct

    return np.frombuffer(hashlib.shake_256(key + struct.pack("<Q", index) + tag).digest(length), np.uint8)


@pytest.mark.parametrize("form", [d.FORM_TC, d.FORM_DP4A])
def test_mixed_device_coins(engine, form):
    """Keypair / encaps requests without coins draw them inside the persistent kernel; the
    coins are recomputed independently (hashlib) and checked through the batched calls."""
    rng = np.random.default_rng(11)
    key, first = bytes(rng.integers(0, 256, 32, dtype=np.uint8)), 5000
    items = []
    for scheme in SCHEMES:
        z = d.sizes(scheme)
        pk_base, _ = engine.keypair(scheme, engine.coins(3, z["kp_coins"], "base", first=scheme), d.FORM_TC)
        for k in range(3):
            items.append((scheme, 0, None, None, torch.empty(z["pk"], dtype=torch.uint8, device="cuda"),
                          torch.empty(z["sk"], dtype=torch.uint8, device="cuda")))
            items.append((scheme, 1, None, torch.from_numpy(pk_base[k].copy()).cuda(),
                          torch.empty(z["ct"], dtype=torch.uint8, device="cuda"),
                          torch.empty(z["ss"], dtype=torch.uint8, device="cuda")))
    items = [items[j] for j in rng.permutation(len(items))]
    expect = []  # the coin index is the position in the submitted list
    for pos, (scheme, op, _, in1, o0, o1) in enumerate(items):
        z = d.sizes(scheme)
        tag, length = (b"kp", z["kp_coins"]) if op == 0 else (b"enc", z["enc_coins"])
        c = _host_coins(key, first + pos, tag, length)[None].copy()
        if op == 0:
            r0, r1 = engine.keypair(scheme, c, d.FORM_TC)
        else:
            r0, r1 = engine.enc(scheme, in1.cpu().numpy()[None], c, d.FORM_TC)
        expect.append(((o0, r0[0]), (o1, r1[0])))
    engine.mixed(items, form, coin_key=key, coin_first=first)
    engine.sync()
    torch.cuda.synchronize()
    for pairs in expect:
        for got, ref in pairs:
            assert (got.cpu().numpy() == ref).all()


def test_mixed_null_inputs_rejected(engine):
    z = d.sizes(d.SABER)
    opk = torch.empty(z["pk"], dtype=torch.uint8, device="cuda")
    osk = torch.empty(z["sk"], dtype=torch.uint8, device="cuda")
    oss = torch.empty(z["ss"], dtype=torch.uint8, device="cuda")
    sk = torch.zeros(z["sk"], dtype=torch.uint8, device="cuda")
    with pytest.raises(d.DpkemError) as e:  # no coins and no key
        engine.mixed([(d.SABER, 0, None, None, opk, osk)], d.FORM_TC)
    assert e.value.status == d.kem.EINVAL
    with pytest.raises(d.DpkemError) as e:  # decaps needs its ciphertext even with a key
        engine.mixed([(d.SABER, 2, None, sk, oss, None)], d.FORM_TC, coin_key=bytes(32))
    assert e.value.status == d.kem.EINVAL


@pytest.mark.parametrize("warp", [0, 1 << 20])
@pytest.mark.parametrize("form", [d.FORM_TC, d.FORM_DP4A])
def test_mixed_warp_tasks(engine, oracle_check_items, warp, form):
    """The sponge stages of a mixed batch as thread tasks (a thread per instance) or as warp
    tasks (a warp per instance and role; mixed_warp_max), every scheme and op, tampered
    decaps included: equal to the batched calls and, on every fifth request, to the oracle."""
    from dpcrypto_b200 import kem

    with kem.knobs(mixed_warp_max=warp):
        items, expect = _mixed_case(engine, 7, 5, form)
        engine.mixed(items, form)
        engine.sync()
        torch.cuda.synchronize()
    for pairs in expect:
        for got, ref in pairs:
            assert torch.equal(got, ref)
    assert oracle_check_items(items, stride=5) >= 20


@pytest.mark.parametrize("warp", [0, 1 << 20])
def test_mixed_warp_tasks_device_coins(engine, oracle, warp):
    """Keypair requests without coins draw them inside the kernel; with warp tasks one lane
    draws them for its warp.  With key 00..1F the stream is the oracle's coins(i, "kp"), so the
    key pairs must equal the oracle's for those coins."""
    from dpcrypto_b200 import kem

    key = bytes(range(32))
    with kem.knobs(mixed_warp_max=warp):
        items, outs = [], []
        for scheme in (d.FRODO976, d.SABER):
            z = d.sizes(scheme)
            for i in range(3):
                opk = torch.empty(z["pk"], dtype=torch.uint8, device="cuda")
                osk = torch.empty(z["sk"], dtype=torch.uint8, device="cuda")
                items.append((scheme, 0, None, None, opk, osk))
                outs.append((scheme, len(items) - 1, opk, osk))
        engine.mixed(items, d.FORM_TC, coin_key=key, coin_first=40)
        engine.sync()
        torch.cuda.synchronize()
    for scheme, pos, opk, osk in outs:
        z = d.sizes(scheme)
        kc = oracle.coins(1, z["kp_coins"], "kp", first=40 + pos)
        pk_o, sk_o = oracle.keypair(scheme, kc)
        assert (opk.cpu().numpy() == pk_o[0]).all() and (osk.cpu().numpy() == sk_o[0]).all()
