"""Wire format and shared-memory ring protocol (include/dpkem_wire.h) without a GPU.

The ring tests stand in for the GPU with a fake server that answers each request frame
with a response frame of the right size whose payload bytes are the request id's low
byte; the protocol (wrap-around with PAD frames, flow control in both directions, order,
cross-process visibility) is the same code the frame server runs."""
import multiprocessing as mp
import os
import tempfile

import numpy as np
import pytest

import dpcrypto_b200 as d
from dpcrypto_b200 import frames as F
from dpcrypto_b200 import kem as K

SCHEMES = [d.FRODO976, d.LIGHTSABER, d.SABER, d.FIRESABER]


def _payload(scheme, op, n, rng):
    z = d.sizes(scheme)
    r = lambda k: rng.integers(0, 256, (n, k), dtype=np.uint8)  # noqa: E731
    if op == 0:
        return {"coins": r(z["kp_coins"])}
    if op == 1:
        return {"coins": r(z["enc_coins"]), "pk": r(z["pk"])}
    return {"ct": r(z["ct"]), "sk": r(z["sk"])}


@pytest.mark.parametrize("scheme", SCHEMES)
def test_frame_layout(scheme):
    z = d.sizes(scheme)
    for op in range(3):
        rq, rs = F.frame_bytes(scheme, op)
        assert rq % 32 == 0 and rs % 32 == 0
        for resp in (False, True):
            secs = F.sections(scheme, op, resp)
            for name, off, length in secs:
                assert off % 16 == 0
                assert off + length <= (rs if resp else rq)
            end = secs[-1][1] + secs[-1][2]
            assert (rs if resp else rq) - end < 32 + 16
    if scheme == d.FRODO976:  # header + 24-byte coins padded to 32 + pk, rounded up to 32
        assert F.frame_bytes(scheme, 1) == (15712, 15808)
        assert F.frame_bytes(scheme, 0) == (96, 32 + z["pk"] + z["sk"] + 16)


def test_encode_scan_and_headers():
    rng = np.random.default_rng(1)
    blocks, n_total, resp_total = [], 0, 0
    for scheme in SCHEMES:
        for op in range(3):
            n = 3
            blocks.append(F.encode(scheme, op, np.arange(n) + 100 * scheme + 10 * op, **_payload(scheme, op, n, rng)))
            n_total += n
            resp_total += n * F.frame_bytes(scheme, op)[1]
    blocks.insert(3, F.pad_frame(96))
    blk = np.concatenate(blocks)
    assert F.scan(blk) == (n_total, len(blk), resp_total)
    h = F.headers(blk)
    assert (h["magic"] == F.PAD).sum() == 1
    real = h[h["magic"] == F.MAGIC]
    assert len(real) == n_total and (real["version"] == 1).all()
    # prefix of k frames
    k, used, _ = F.scan(blk, max_frames=4)
    assert k == 4 and F.scan(blk[:used])[0] == 4
    # payload sections sit where `sections` says
    one = F.encode(d.SABER, 1, [7], coins=np.full((1, 32), 5, np.uint8), pk=np.full((1, 992), 9, np.uint8))
    (_, o1, l1), (_, o2, l2) = F.sections(d.SABER, 1, False)
    assert (one[o1:o1 + l1] == 5).all() and (one[o2:o2 + l2] == 9).all()


def test_scan_rejects_bad_frames():
    rng = np.random.default_rng(2)
    good = F.encode(d.SABER, 2, [1, 2], **_payload(d.SABER, 2, 2, rng))
    size = F.frame_bytes(d.SABER, 2)[0]
    cases = []
    for field, value in (("magic", 0x12345678), ("version", 2), ("scheme", 5), ("scheme", 9), ("op", 3),
                         ("frame_bytes", size + 32)):
        bad = good.copy()
        h = bad[:32].view(F.HDR_DTYPE)
        h[field] = value
        cases.append(bad)
    cases.append(good[:-32])  # truncated
    cases.append(np.concatenate([good, F.pad_frame(64)[:48]]))  # PAD running past the end
    for bad in cases:
        with pytest.raises(K.DpkemError) as e:
            F.scan(bad)
        assert e.value.status == K.EINVAL


def _fake_answer(ring, a):
    """Answer acquired request frames: header copied, payload = id's low byte."""
    req = ring.request_view(a["req_off"], a["req_bytes"])
    out = ring.response_view(a["resp_off"], a["resp_bytes"])
    pos = 0
    for h in F.headers(req):
        size = F.frame_bytes(int(h["scheme"]), int(h["op"]))[1]
        r = np.zeros(size, np.uint8)
        rh = r[:32].view(F.HDR_DTYPE)
        rh["magic"], rh["version"], rh["scheme"], rh["op"] = F.MAGIC, 1, h["scheme"], h["op"]
        rh["id"], rh["frame_bytes"] = h["id"], size
        r[32:] = int(h["id"]) & 0xFF
        out[pos:pos + size] = r
        pos += size
    assert pos == a["resp_bytes"]


def _client_loop(ring, batches, serve):
    """Push every batch (retrying while the ring is full), pop everything, in order.
    With serve=True this process also plays the server, a few frames at a time."""
    total = sum(len(F.headers(b)) for b in batches)
    ids, pending = [], list(batches)
    while pending or len(ids) < total:
        if pending:
            took = ring.push(pending[0])
            pending[0] = pending[0][took:]
            if len(pending[0]) == 0:
                pending.pop(0)
        if serve:
            a = ring.acquire(max_frames=7)
            if a is not None:
                _fake_answer(ring, a)
                ring.release(a)
        blk, count = ring.pop()
        pos = 0
        assert count == (len(F.headers(blk)) if len(blk) else 0)
        for h in (F.headers(blk) if len(blk) else []):
            size = int(h["frame_bytes"])
            assert h["magic"] == F.MAGIC
            assert (blk[pos + 32:pos + size] == (int(h["id"]) & 0xFF)).all()
            ids.append(int(h["id"]))
            pos += size
    return ids


def _batches(seed, count):
    rng = np.random.default_rng(seed)
    out, next_id = [], 0
    for _ in range(count):
        scheme = int(rng.choice(SCHEMES[1:]))  # Saber frames: small enough for a small ring
        op = int(rng.integers(0, 3))
        n = int(rng.integers(1, 5))
        out.append(F.encode(scheme, op, np.arange(next_id, next_id + n), **_payload(scheme, op, n, rng)))
        next_id += n
    return out, next_id


def test_ring_in_process_wraps_and_keeps_order():
    with tempfile.TemporaryDirectory() as tmp:
        ring = F.Ring(os.path.join(tmp, "ring"), capacity=16384)
        batches, total = _batches(3, 120)
        ids = _client_loop(ring, batches, serve=True)
        assert ids == list(range(total))
        assert ring.counter("served") == total
        assert ring.counter("req_head") == ring.counter("req_tail")
        assert ring.counter("req_tail") > 3 * ring.capacity  # wrapped several times
        ring.close()


def test_ring_push_takes_what_fits():
    with tempfile.TemporaryDirectory() as tmp:
        ring = F.Ring(os.path.join(tmp, "ring"), capacity=4096)
        rng = np.random.default_rng(4)
        dec = F.encode(d.SABER, 2, [0], **_payload(d.SABER, 2, 1, rng))  # 3424 B
        assert ring.push(dec) == len(dec)
        kps = F.encode(d.SABER, 0, np.arange(1, 8), **_payload(d.SABER, 0, 7, rng))  # 7 x 128 B
        assert ring.push(kps) == 5 * 128  # 672 B left: a prefix of 5 whole frames, then a PAD
        assert ring.counter("req_tail") == ring.capacity  # the last 32 B closed by a PAD
        assert ring.push(dec) == 0  # no room until the server consumes
        big = F.encode(d.FRODO976, 1, [9], **_payload(d.FRODO976, 1, 1, rng))  # larger than the ring
        with pytest.raises(K.DpkemError):
            ring.push(big)
        ring.close()


def test_ring_no_deadlock_on_large_frames():
    """A frame that fits neither before the end nor after a PAD in the current free space
    still gets through: the writer closes the end with a PAD first."""
    with tempfile.TemporaryDirectory() as tmp:
        ring = F.Ring(os.path.join(tmp, "ring"), capacity=8192)
        rng = np.random.default_rng(6)
        small = F.encode(d.FIRESABER, 0, [0], **_payload(d.FIRESABER, 0, 1, rng))  # 128 B, 4384-B response
        big = F.encode(d.FIRESABER, 2, [1], **_payload(d.FIRESABER, 2, 1, rng))  # 4544 B
        ids = _client_loop(ring, [small] * 30 + [big, small, big], serve=True)
        assert len(ids) == 33
        ring.close()


def _fake_server_proc(path, n_expected):
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from dpcrypto_b200 import frames as F2

    ring = F2.Ring(path)
    served = 0
    while not ring.counter("stop"):
        a = ring.acquire(max_frames=5)
        if a is None:
            continue
        _fake_answer(ring, a)
        ring.release(a)
        served += a["n_frames"]
    ring.close()
    raise SystemExit(0 if served == n_expected else 3)


def test_ring_across_processes():
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "ring")
        ring = F.Ring(path, capacity=16384)
        batches, total = _batches(5, 80)
        p = mp.get_context("spawn").Process(target=_fake_server_proc, args=(path, total))
        p.start()
        try:
            ids = _client_loop(ring, batches, serve=None)
            assert ids == list(range(total))
        finally:
            ring.stop()
            p.join(60)
        assert p.exitcode == 0
        ring.close()
