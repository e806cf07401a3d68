"""Wire-format frames on the GPU (include/dpkem_wire.h): dpkem_frames_run against the
batched entry points and the oracle, and the frame server process fed through a
shared-memory ring by this (client) process."""
import os
import subprocess
import sys
import tempfile
import time

import numpy as np
import pytest

import dpcrypto_b200 as d
from dpcrypto_b200 import frames as F

pytestmark = pytest.mark.gpu
SCHEMES = [d.FRODO976, d.FRODO976AES, d.LIGHTSABER, d.SABER, d.FIRESABER]
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _case(engine, oracle, per_kind, seed, form=d.FORM_TC):
    """A shuffled block with per_kind requests of each (scheme, op), PAD frames between
    some of them; returns (block, expected {id: {section: bytes}}, kinds {id: (scheme, op)})."""
    rng = np.random.default_rng(seed)
    frames, expected, kinds, next_id = [], {}, {}, 0
    for scheme in SCHEMES:
        z = d.sizes(scheme)
        n = per_kind
        kc = oracle.coins(2 * n, z["kp_coins"], "kp", first=seed * 1000)
        ec = oracle.coins(n, z["enc_coins"], "enc", first=seed * 1000)
        pk, sk = engine.keypair(scheme, kc, d.FORM_DP4A)
        ct, ss = engine.enc(scheme, pk[n:], ec, d.FORM_DP4A)
        bad = ct.copy()
        bad[::2, 5] ^= 0x10  # half of the decaps tampered: implicit rejection
        ss_dec = engine.dec(scheme, bad, sk[n:], d.FORM_DP4A)
        for i in range(n):
            frames.append(F.encode(scheme, 0, [next_id], coins=kc[i:i + 1]))
            expected[next_id], kinds[next_id] = {"pk": pk[i], "sk": sk[i]}, (scheme, 0)
            next_id += 1
            frames.append(F.encode(scheme, 1, [next_id], coins=ec[i:i + 1], pk=pk[n + i:n + i + 1]))
            expected[next_id], kinds[next_id] = {"ct": ct[i], "ss": ss[i]}, (scheme, 1)
            next_id += 1
            frames.append(F.encode(scheme, 2, [next_id], ct=bad[i:i + 1], sk=sk[n + i:n + i + 1]))
            expected[next_id], kinds[next_id] = {"ss": ss_dec[i]}, (scheme, 2)
            next_id += 1
    order = rng.permutation(len(frames))
    blocks = []
    for k, j in enumerate(order):
        blocks.append(frames[j])
        if k % 7 == 3:
            blocks.append(F.pad_frame(64))
    return np.concatenate(blocks), expected, kinds


def _check(resp, expected, kinds, order=None):
    ids, pos = [], 0
    for h in F.headers(resp):
        assert h["magic"] == F.MAGIC and h["status"] == 0 and h["version"] == 1
        i = int(h["id"])
        scheme, op = kinds[i]
        assert (int(h["scheme"]), int(h["op"])) == (scheme, op)
        size = F.frame_bytes(scheme, op)[1]
        assert int(h["frame_bytes"]) == size
        for name, off, length in F.sections(scheme, op, response=True):
            assert (resp[pos + off:pos + off + length] == expected[i][name]).all(), (i, name)
        ids.append(i)
        pos += size
    assert pos == len(resp)
    return ids


@pytest.mark.parametrize("form", [d.FORM_TC, d.FORM_DP4A, d.FORM_INT32])
def test_frames_run_mixed_block(engine, oracle, form):
    blk, expected, kinds = _case(engine, oracle, 3, seed=1)
    req_ids = [int(h["id"]) for h in F.headers(blk) if h["magic"] == F.MAGIC]
    resp = F.run(engine, blk, form)
    assert _check(resp, expected, kinds) == req_ids  # responses in request order


def test_frames_run_matches_oracle(engine, oracle):
    scheme, n = d.FRODO976, 2
    z = d.sizes(scheme)
    kc, ec = oracle.coins(n, 64, "kp", first=7), oracle.coins(n, 24, "enc", first=7)
    pk_o, sk_o = oracle.keypair(scheme, kc, threads=2)
    ct_o, ss_o = oracle.enc(scheme, pk_o, ec, threads=2)
    blk = np.concatenate([F.encode(scheme, 0, [1, 2], coins=kc), F.encode(scheme, 1, [3, 4], coins=ec, pk=pk_o),
                          F.encode(scheme, 2, [5, 6], ct=ct_o, sk=sk_o)])
    resp = F.run(engine, blk)
    k0, k1 = F.frame_bytes(scheme, 0)[1] * 2, F.frame_bytes(scheme, 1)[1] * 2
    r0, r1, r2 = F.decode(resp[:k0], scheme, 0), F.decode(resp[k0:k0 + k1], scheme, 1), F.decode(resp[k0 + k1:], scheme, 2)
    assert (r0["pk"] == pk_o).all() and (r0["sk"] == sk_o).all() and list(r0["id"]) == [1, 2]
    assert (r1["ct"] == ct_o).all() and (r1["ss"] == ss_o).all()
    assert (r2["ss"] == ss_o).all() and z["ss"] == r2["ss"].shape[1]


def test_frames_run_pipelined_small_budget(oracle):
    """Enough frames for several pipeline chunks, and a budget that forces chunks to reuse
    their arena regions in turn."""
    eng = d.Engine(0, hbm_budget=24 << 20)
    try:
        blk, expected, kinds = _case(eng, oracle, 120, seed=2)
        req_ids = [int(h["id"]) for h in F.headers(blk) if h["magic"] == F.MAGIC]
        resp = F.run(eng, blk)
        assert _check(resp, expected, kinds) == req_ids
    finally:
        eng.close()


def test_frame_server_process(engine, oracle):
    """The frame server as its own process, fed through a shared-memory ring."""
    blk, expected, kinds = _case(engine, oracle, 40, seed=3)
    req_ids = [int(h["id"]) for h in F.headers(blk) if h["magic"] == F.MAGIC]
    shm = "/dev/shm" if os.path.isdir("/dev/shm") else tempfile.gettempdir()
    path = os.path.join(shm, f"dpkem-test-{os.getpid()}.ring")
    ring = F.Ring(path, capacity=8 << 20)
    proc = subprocess.Popen([sys.executable, "-m", "dpcrypto_b200.frame_server", "--ring", path, "--max-frames", "64"],
                            cwd=ROOT)
    try:
        got, n_got, pending, deadline = [], 0, blk, time.time() + 120
        while n_got < len(req_ids):
            assert time.time() < deadline and proc.poll() is None
            if len(pending):
                pending = pending[ring.push(pending):]
            r, count = ring.pop()
            if count:
                got.append(r.copy())
                n_got += count
        resp = np.concatenate(got)
        assert _check(resp, expected, kinds) == req_ids
        assert proc.poll() is None  # still serving
    finally:
        ring.stop()
        rc = proc.wait(timeout=60)
        ring.close()
        os.unlink(path)
    assert rc == 0
