"""KEM service (dpkem_service_*): one long-lived launch that admits requests while it runs.
Every request's outputs must equal the batched calls' on the same inputs (alone vs in the
mix), a stride sample also the CPU oracle's; admission must be live (ring slots and scratch
bytes), idle launches must end and be relaunched, and every ticket must come back once."""
import time

import numpy as np
import pytest
import torch

import dpcrypto_b200 as d
from test_gpu_mixed import _host_coins, _mixed_case

pytestmark = pytest.mark.gpu


def _check(expect):
    torch.cuda.synchronize()
    for pairs in expect:
        for got, ref in pairs:
            assert torch.equal(got, ref)


def _submit_all(svc, items, chunk):
    """Submits items in chunks while the service runs; returns every ticket issued."""
    tickets = []
    for a in range(0, len(items), chunk):
        part = items[a:a + chunk]
        while part:
            acc, first = svc.submit(part)
            tickets += list(range(first, first + acc))
            part = part[acc:]
            if part:
                svc.poll()
                time.sleep(1e-4)
        time.sleep(2e-3)
    return tickets


@pytest.mark.parametrize("form", [d.FORM_TC, d.FORM_DP4A, d.FORM_INT32])
def test_service_equals_batched(engine, oracle_check_items, form):
    items, expect = _mixed_case(engine, 4, 11, form)
    with d.Service(engine, form) as svc:
        tickets = _submit_all(svc, items, 7)
        svc.drain()
        st = svc.stats()
        assert st["submitted"] == st["completed"] == len(items)
        assert tickets == list(range(len(items)))
    _check(expect)
    assert oracle_check_items(items, 5) >= 10


@pytest.mark.parametrize("warp_max", [0, 1 << 30])
def test_service_thread_and_warp_gangs(engine, warp_max):
    """Thread-level stages as one thread per instance only, and as a warp per instance only."""
    items, expect = _mixed_case(engine, 3, 12, d.FORM_TC)
    with d.Service(engine, d.FORM_TC, warp_max=warp_max, saber_ctas=16) as svc:
        _submit_all(svc, items, len(items))
        svc.drain()
    _check(expect)


def test_service_poll_returns_each_ticket_once(engine):
    items, expect = _mixed_case(engine, 2, 13, d.FORM_TC)
    seen = []
    with d.Service(engine, d.FORM_TC) as svc:
        for a in range(0, len(items), 5):
            acc, first = svc.submit(items[a:a + 5])
            assert acc == len(items[a:a + 5]) and first == a
            seen += svc.poll().tolist()
        t0 = time.time()
        while len(seen) < len(items) and time.time() - t0 < 30:
            seen += svc.poll().tolist()
            time.sleep(1e-4)
    assert sorted(seen) == list(range(len(items)))
    _check(expect)


def test_service_admission_is_live(engine):
    """Ring slots and scratch bytes bound the requests in flight; room comes back as they
    complete.  Three FrodoKEM records of scratch admit three FrodoKEM requests at a time."""
    items, expect = _mixed_case(engine, 4, 14, d.FORM_TC)
    frodo = [it for it in items if it[0] == d.FRODO976][:6]
    frodo_expect = [e for it, e in zip(items, expect) if it[0] == d.FRODO976][:6]
    with d.Service(engine, d.FORM_TC, scratch_bytes=3 * 31744 + 1000) as svc:
        acc, first = svc.submit(frodo)
        assert (acc, first) == (3, 0)
        svc.drain()
        acc, first = svc.submit(frodo[3:])
        assert (acc, first) == (3, 3)
        svc.drain()
    _check(frodo_expect)
    items, expect = _mixed_case(engine, 6, 16, d.FORM_TC)  # 90 requests
    with d.Service(engine, d.FORM_TC, max_inflight=64) as svc:  # 64 ring slots
        acc, first = svc.submit(items)
        assert (acc, first) == (64, 0)
        svc.drain()
        acc, first = svc.submit(items[64:])
        assert (acc, first) == (len(items) - 64, 64)
        svc.drain()
    _check(expect)


def test_service_idle_exit_and_relaunch(engine):
    items, expect = _mixed_case(engine, 1, 15, d.FORM_TC)
    with d.Service(engine, d.FORM_TC, idle_ms=50) as svc:
        svc.submit(items)
        svc.drain()
        time.sleep(0.5)
        st = svc.stats()
        assert st["launches"] == 1 and not st["running"]
        for pairs in expect:
            for got, _ in pairs:
                got.zero_()
        torch.cuda.synchronize()
        acc, first = svc.submit(items)
        assert acc == len(items) and first == len(items)
        svc.drain()
        assert svc.stats()["launches"] == 2
    _check(expect)


def test_service_device_coins(engine):
    """Keypair / encaps requests without coins draw SHAKE256(key || LE64(ticket) || tag)."""
    key = bytes(range(100, 132))
    rows = []
    for scheme in (d.FRODO976, d.SABER):
        z = d.sizes(scheme)
        pk_in, _ = engine.keypair(scheme, torch.from_numpy(_host_coins(b"\x07" * 32, scheme, b"x", z["kp_coins"])
                                                            .copy()).cuda().reshape(1, -1), d.FORM_TC)
        rows.append((scheme, 0, None, None, torch.empty(z["pk"], dtype=torch.uint8, device="cuda"),
                     torch.empty(z["sk"], dtype=torch.uint8, device="cuda")))
        rows.append((scheme, 1, None, pk_in[0], torch.empty(z["ct"], dtype=torch.uint8, device="cuda"),
                     torch.empty(z["ss"], dtype=torch.uint8, device="cuda")))
    with d.Service(engine, d.FORM_TC, coin_key=key) as svc:
        acc, first = svc.submit(rows)
        assert acc == len(rows) and first == 0
        svc.drain()
    for t, (scheme, op, _, pk, o0, o1) in enumerate(rows):
        z = d.sizes(scheme)
        if op == 0:
            c = torch.from_numpy(_host_coins(key, t, b"kp", z["kp_coins"]).copy()).cuda().reshape(1, -1)
            pk_ref, sk_ref = engine.keypair(scheme, c, d.FORM_DP4A)
            assert torch.equal(o0, pk_ref[0]) and torch.equal(o1, sk_ref[0])
        else:
            c = torch.from_numpy(_host_coins(key, t, b"enc", z["enc_coins"]).copy()).cuda().reshape(1, -1)
            ct_ref, ss_ref = engine.enc(scheme, pk.reshape(1, -1), c, d.FORM_DP4A)
            assert torch.equal(o0, ct_ref[0]) and torch.equal(o1, ss_ref[0])
